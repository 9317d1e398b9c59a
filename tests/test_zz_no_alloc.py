"""The allocation-free sphere fill-fraction entry point.

Callers that cannot allocate device memory while they rasterise a sphere (a
scene-building thread next to a thread capturing a CUDA graph, a real-time
loop that must not enter the allocator, a process whose device memory is
owned by another framework's pool) use fdtd_b200_sphere_fractions_noalloc,
which stages its results in a fixed device array instead of cudaMalloc.  Its
output must equal that of the allocating path the sphere rasteriser uses,
call after call, since the staging array is shared and keeps the previous
call's contents; the calls must leave the device's free memory and the
library's memory cache unchanged; and a call made while another thread
captures a CUDA graph in the global capture mode must neither fail nor
break that capture.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes as C
import threading

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


def test_noalloc_calls_allocate_nothing():
    import torch

    lib = rb.load()
    noalloc = _bind(lib, "fdtd_b200_sphere_fractions_noalloc")
    assert _call(noalloc, (8.0, 8.0, 8.0), 3.0, (4, 4, 4, 9, 9, 9))[0] == 0  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    cached0 = rb.cached_bytes()
    boxes = [((30.2, 29.9, 31.4), 20.5, (9, 9, 10, 44, 43, 43)),
             ((5.1, 6.3, 7.7), 2.2, (2, 3, 4, 7, 7, 7)),
             ((40.0, 41.0, 39.0), 14.0, (25, 26, 24, 30, 31, 32))]
    for centre, radius, box in boxes:
        rc, f, n2 = _call(noalloc, centre, radius, box)
        assert rc == 0, rb.last_error()
        assert np.all(np.isfinite(f)) and np.all(np.isfinite(n2))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert rb.cached_bytes() == cached0


def test_noalloc_beside_a_global_mode_capture_on_another_thread():
    import torch

    lib = rb.load()
    allocating = _bind(lib, "rfb_sphere_fractions")
    noalloc = _bind(lib, "fdtd_b200_sphere_fractions_noalloc")
    centre, radius, box = (12.4, 13.1, 11.8), 6.3, (5, 6, 4, 15, 14, 16)
    assert _call(noalloc, centre, radius, box)[0] == 0  # set-up call, before any capture
    rc_a, f_a, n_a = _call(allocating, centre, radius, box)
    assert rc_a == 0, rb.last_error()

    x = torch.arange(1024, dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    g = torch.cuda.CUDAGraph()
    capturing, called = threading.Event(), threading.Event()
    out = {}

    def other_thread():
        capturing.wait(timeout=60)
        out["res"] = _call(noalloc, centre, radius, box)
        out["err"] = rb.last_error()
        called.set()

    t = threading.Thread(target=other_thread)
    t.start()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side, capture_error_mode="global"):
            y.copy_(x * 2.0)
            capturing.set()
            assert called.wait(timeout=60), "the allocation-free call did not return during the capture"
            y.add_(1.0)
    t.join(timeout=60)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, x * 2.0 + 1.0)
    rc_b, f_b, n_b = out["res"]
    assert rc_b == 0, out["err"]
    assert np.array_equal(f_a, f_b)
    assert np.array_equal(n_a, n_b)
