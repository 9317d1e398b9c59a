"""Batches of independent scenes advanced together (fdtd_b200_batch_*).

Every scene of a batch must give exactly the probe series and spectra of
its own single-scene session (same kernels, same arithmetic), in FP32 and
FP64; FP64 batch scenes equal the CPU oracle bit for bit; the batch rejects
what it cannot run."""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import scenes
from tests.cases import CASES, scene_run_config

pytestmark = pytest.mark.gpu


def _small_batch(precision, n=6, steps=60):
    return scenes.c4(seed=11, n_scenes=n, precision=precision, n_steps=steps, lo=20, hi=44, npml=4)


def _single(w):
    setup = scenes.scene_setup(w)
    sim = rb.Sim(scenes.run_config(w), setup.ptr if setup else None, None)
    try:
        sim.advance(w.n_steps)
        return sim.probes(), sim.dft()
    finally:
        sim.close()


@pytest.mark.parametrize("precision", [rb.FP32, rb.FP64], ids=["fp32", "fp64"])
def test_batch_scenes_equal_their_single_sessions(precision):
    ws = _small_batch(precision)
    setups = [scenes.scene_setup(w) for w in ws]
    b = rb.Batch([scenes.run_config(w) for w in ws], [s.ptr if s else None for s in setups])
    try:
        info = b.info()
        assert info.scenes == len(ws) and info.launches_per_step <= 5
        b.advance(17)
        b.advance(ws[0].n_steps - 17)
        for q, w in enumerate(ws):
            td, dft = _single(w)
            assert np.array_equal(b.probes(q), td), q
            assert np.array_equal(b.dft(q), dft), q
    finally:
        b.close()


@pytest.mark.parametrize("mode", [2, 3])
def test_batch_plans_agree(mode, monkeypatch):
    """Forced plans (tile origins from 0 / shifted to the slab edges) give
    identical results."""
    ws = _small_batch(rb.FP32, n=4, steps=40)
    setups = [scenes.scene_setup(w) for w in ws]
    rcs = [scenes.run_config(w) for w in ws]
    ref = rb.Batch(rcs, [s.ptr if s else None for s in setups])
    ref.advance(40)
    want = [ref.probes(q) for q in range(len(ws))]
    ref.close()
    monkeypatch.setenv("RFSYN_FDTD_PLAN", f"8,4,32,16,{mode}")
    b = rb.Batch(rcs, [s.ptr if s else None for s in setups])
    assert b.info().mode == mode
    b.advance(40)
    for q in range(len(ws)):
        assert np.array_equal(b.probes(q), want[q]), q
    b.close()


def test_batch_fp64_equals_oracle():
    """Boundary cases of tests/cases.py without a y / z wrap, batched
    together: bit-equal to the CPU oracle."""
    names = ["cpml_materials", "pec_boundary_sources", "periodic_x_cpml"]
    steps = min(CASES[n].n_steps for n in names)
    rcs, setups, ctxs, keep, wants = [], [], [], [], []
    for n in names:
        s = copy.deepcopy(CASES[n])
        s.n_steps = steps
        wants.append(oracle.run_oracle(s)["td"])
        rcs.append(scene_run_config(s, rb.FP64, rb.FUSED))
        cs = s.to_c()
        keep.append(cs)
        setups.append(oracle.device_setup())
        ctxs.append(C.cast(C.pointer(cs), C.c_void_p))
    b = rb.Batch(rcs, setups, ctxs)
    b.advance(steps)
    for q, n in enumerate(names):
        assert np.array_equal(b.probes(q), wants[q]), n
    b.close()


def test_batch_rejects_unsupported():
    w = _small_batch(rb.FP32, n=2, steps=10)
    rc0 = scenes.run_config(w[0])
    # a y-periodic scene: its end tiles' halos wrap
    w[1].periodic = 2
    with pytest.raises(RuntimeError, match="wraps"):
        rb.Batch([rc0, scenes.run_config(w[1])])
    # mixed precision
    w[1].periodic = 0
    w[1].precision = rb.FP64
    with pytest.raises(RuntimeError, match="precision"):
        rb.Batch([rc0, scenes.run_config(w[1])])
    # advancing past the step count
    b = rb.Batch([rc0])
    b.advance(10)
    with pytest.raises(RuntimeError, match="past the configured step count"):
        b.advance(1)
    b.close()


def test_members_built_on_threads_match_one_thread(monkeypatch):
    ws = _small_batch(rb.FP32, n=8, steps=40)

    def run():
        setups = [scenes.scene_setup(w) for w in ws]
        b = rb.Batch([scenes.run_config(w) for w in ws], [s.ptr if s else None for s in setups])
        try:
            b.advance(40)
            return [b.probes(q) for q in range(len(ws))]
        finally:
            b.close()

    monkeypatch.setenv("RFSYN_FDTD_CREATE_THREADS", "1")
    one = run()
    monkeypatch.setenv("RFSYN_FDTD_CREATE_THREADS", "8")
    many = run()
    assert all(np.array_equal(x, y) for x, y in zip(one, many))
    # the error names the lowest-numbered failing scene, as one thread would
    bad = copy.deepcopy(ws)
    for q in (5, 2, 6):
        bad[q].sources[0]["i"] = bad[q].nx + 3
    with pytest.raises(RuntimeError, match="batch scene 2: source 0 outside the grid"):
        rb.Batch([scenes.run_config(w) for w in bad])
