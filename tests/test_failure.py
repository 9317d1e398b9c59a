"""Failure detection without a GPU fault.

Every sweep waits on its tensor copies with a bounded wait and reports a
stalled copy as an error the host returns; these tests make that wait run
out on purpose -- an mbarrier armed for a copy that is never issued -- and
check that the status comes back and the device stays usable.  Host-side
failures (bad arguments, rejected scenes) are covered by the ABI tests."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from tests.cases import CASES, run_device


def _selftest(limit):
    lib = rb.load()
    f = lib.fdtd_b200_selftest_bounded_wait
    f.restype = C.c_int
    f.argtypes = [C.c_longlong, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    timed_out, cycles = C.c_int(-1), C.c_longlong(0)
    rc = f(limit, C.byref(timed_out), C.byref(cycles))
    return rc, timed_out.value, cycles.value


@pytest.mark.parametrize("limit", [0, -5, 5_000_000_000])
def test_selftest_rejects_limits_before_device_work(limit):
    rc, _, _ = _selftest(limit)
    assert rc == -1
    assert "limit" in rb.last_error()


@pytest.mark.gpu
def test_bounded_wait_gives_up_and_device_stays_usable():
    rc, timed_out, cycles = _selftest(200_000_000)     # ~0.1 s at B200 clocks
    assert rc == 0, rb.last_error()
    assert timed_out == 1
    assert 200_000_000 <= cycles < 2_000_000_000
    # the context still runs a simulation bit-exactly
    s = CASES["cpml_materials"]
    assert np.array_equal(run_device(s, rb.FP64, rb.FUSED)["td"], oracle.run_oracle(s)["td"])
