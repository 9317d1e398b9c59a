"""Host-side fault injection: a forced device-allocation failure.

RFSYN_FDTD_FAIL_ALLOC=n makes the n-th device allocation that the creating
thread makes inside a single-scene engine creation (field buffers, CPML,
scene upload, plan, graphs) report out-of-memory without calling the driver
(no device fault).  Creating a small scene with n = 1, 2, ... walks every
allocation of engine creation (the host-side scene building before it, and
the sphere rasteriser's staging, are not walked): each attempt must fail
with an error the host reads, free what it had built and leave the device
usable, until n passes the number of
allocations and creation succeeds.  The scene built afterwards, partly on
memory the failed attempts released, gives the same probe series and
spectra bit for bit as before the failures.  Collected late, so a fault
here cannot hide the results of the other files."""
from __future__ import annotations

import numpy as np
import pytest

import rfsyn_b200 as rb
from rfsyn_b200 import scenes

pytestmark = pytest.mark.gpu


def _scene():
    # a box or sphere scene of ~28^3 with CPML, one source, probes and DFT bins
    ws = scenes.c4(seed=12, n_scenes=4, precision=rb.FP32, n_steps=40, lo=26, hi=30, npml=4)
    return next(w for w in ws if w.boxes or w.spheres)


def _create(w):
    setup = scenes.scene_setup(w)
    return rb.Sim(scenes.run_config(w), setup.ptr if setup else None, None), setup


def _run(w):
    sim, _setup = _create(w)
    try:
        sim.advance(w.n_steps)
        return sim.probes(), sim.dft()
    finally:
        sim.close()


def test_every_allocation_of_creation_fails_cleanly(monkeypatch):
    w = _scene()
    td0, dft0 = _run(w)
    failed = 0
    for n in range(1, 200):
        monkeypatch.setenv("RFSYN_FDTD_FAIL_ALLOC", str(n))
        try:
            sim, _setup = _create(w)
        except RuntimeError as exc:
            failed += 1
            assert "fdtd_b200_sim_create failed" in str(exc) and len(rb.last_error()) > 0
            continue
        sim.close()                       # n is past the last allocation
        break
    else:
        pytest.fail("creation kept failing with the hook past 200 allocations")
    monkeypatch.delenv("RFSYN_FDTD_FAIL_ALLOC")
    assert failed >= 10                   # fields, CPML, scene arrays, sources, probes, plan
    td1, dft1 = _run(w)
    assert np.array_equal(td0, td1) and np.array_equal(dft0, dft1)
