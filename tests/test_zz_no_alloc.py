"""The allocation-free sphere fill-fraction entry point.

Callers that cannot allocate device memory while they rasterise a sphere (a
scene-building thread next to a thread capturing a CUDA graph, a real-time
loop that must not enter the allocator, a process whose device memory is
owned by another framework's pool) use fdtd_b200_sphere_fractions_noalloc,
which stages its results in a fixed device array instead of cudaMalloc.  Its
output must equal that of the allocating path the sphere rasteriser uses,
call after call, since the staging array is shared and keeps the previous
call's contents.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import rfsyn_b200 as rb

pytestmark = pytest.mark.gpu
MAX_SAMPLES = 1 << 20


def _bind(lib, name):
    f = getattr(lib, name)
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_double), C.c_double] + [C.c_int] * 6 + [C.POINTER(C.c_double)] * 2
    return f


def _call(fn, centre, radius, box):
    i0, j0, k0, ni, nj, nk = box
    n = 3 * ni * nj * nk
    f = np.full(n, np.nan)
    n2 = np.full(n, np.nan)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rc = fn((C.c_double * 3)(*centre), radius, i0, j0, k0, ni, nj, nk, dp(f), dp(n2))
    return rc, f, n2


def test_noalloc_matches_allocating_path_on_consecutive_calls():
    lib = rb.load()
    allocating = _bind(lib, "rfb_sphere_fractions")
    noalloc = _bind(lib, "fdtd_b200_sphere_fractions_noalloc")
    cases = [
        ((20.3, 18.7, 21.1), 11.6, (5, 4, 6, 33, 31, 32)),   # large box first
        ((9.5, 10.2, 8.8), 4.1, (3, 4, 2, 14, 13, 15)),      # then a smaller one
    ]
    for centre, radius, box in cases:
        rc_a, f_a, n_a = _call(allocating, centre, radius, box)
        rc_b, f_b, n_b = _call(noalloc, centre, radius, box)
        assert rc_a == 0 and rc_b == 0, rb.last_error()
        # FP64, identical kernel: the tolerance of the FP64 tests is equality
        assert np.array_equal(f_a, f_b)
        assert np.array_equal(n_a, n_b)
        assert 0.0 < f_b.sum() and f_b.min() >= 0.0 and f_b.max() <= 1.0


def test_noalloc_rejects_boxes_beyond_its_limit():
    lib = rb.load()
    noalloc = _bind(lib, "fdtd_b200_sphere_fractions_noalloc")
    side = 102  # 3 * 102^3 > 2^20 samples
    assert 3 * side ** 3 > MAX_SAMPLES
    out = np.zeros(1)
    dp = out.ctypes.data_as(C.POINTER(C.c_double))
    rc = noalloc((C.c_double * 3)(50.0, 50.0, 50.0), 10.0, 0, 0, 0, side, side, side, dp, dp)
    assert rc == -1
    assert "exceeds the maximum" in rb.last_error()
