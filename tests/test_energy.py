"""FP64 energy audit of resident fields (fdtd_b200_sim_energy) against the
oracle's restatement of rfsyn's energy loops
(validate_long_term_stability.c:166-209, audit_periodic_energy.c:53-62).

FP64 fields are bit-identical to the oracle's, so the sums differ only by
summation order: relative difference <= 1e-12; maxima are exact.  FP32 fields
carry their own rounding: <= 1e-4 relative."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import scenes
from tests.cases import CASES, scene_run_config, workload_to_scene

pytestmark = pytest.mark.gpu

SUMS = ("electric_j", "magnetic_j", "electric_prev_j", "cross_j")

ENERGY_SCENES = {
    "cpml_materials": CASES["cpml_materials"],
    "periodic_tensor": CASES["periodic_tensor"],
    "c2_56": workload_to_scene(scenes.scaled(scenes.c2(), 56, 90)),
}


def _sim(s, precision, schedule):
    rc = scene_run_config(s, precision, schedule)
    cs = s.to_c()
    needs = bool(s.boxes or s.comps or s.tensors or s.disp or s.spheres or s.tensor3)
    sim = rb.Sim(rc, oracle.device_setup() if needs else None, C.cast(C.pointer(cs), C.c_void_p) if needs else None)
    sim._keep = cs
    return sim


def _x_range(s):
    return s.npml, s.nx - s.npml


@pytest.mark.parametrize("name", list(ENERGY_SCENES))
def test_energy_fp64_matches_oracle(name):
    s = ENERGY_SCENES[name]
    lo, hi = _x_range(s)
    want = oracle.energy_oracle(s, lo, hi)
    sim = _sim(s, rb.FP64, rb.FUSED)
    try:
        sim.advance(s.n_steps)
        got = sim.energy(lo, hi)
        again = sim.energy(lo, hi)
    finally:
        sim.close()
    assert got == again or all(
        (math.isnan(got[k]) and math.isnan(again[k])) or got[k] == again[k] for k in got)  # deterministic
    for k in SUMS:
        assert want[k] > 0.0
        assert abs(got[k] - want[k]) <= 1e-12 * abs(want[k]), (k, got[k], want[k])
    interior = want["interior_e_j"] + want["interior_h_j"]
    assert abs(got["interior_j"] - interior) <= 1e-12 * interior
    assert got["max_abs_e"] == want["max_abs_e"] and got["max_abs_h"] == want["max_abs_h"]
    assert got["nonfinite"] == 0
    assert got["total_j"] == got["electric_j"] + got["magnetic_j"]
    assert got["modified_prev_j"] == got["electric_prev_j"] + got["cross_j"]


def test_energy_fp32_within_bound():
    s = ENERGY_SCENES["c2_56"]
    want = oracle.energy_oracle(s)
    sim = _sim(s, rb.FP32, rb.FUSED)
    try:
        sim.advance(s.n_steps)
        got = sim.energy()
    finally:
        sim.close()
    for k in SUMS:
        assert abs(got[k] - want[k]) <= 1e-4 * abs(want[k]), (k, got[k], want[k])


def test_energy_split_schedule_has_no_previous_step():
    s = CASES["cpml_materials"]
    want = oracle.energy_oracle(s)
    sim = _sim(s, rb.FP64, rb.SPLIT)
    try:
        sim.advance(s.n_steps)
        got = sim.energy()
    finally:
        sim.close()
    assert math.isnan(got["electric_prev_j"]) and math.isnan(got["modified_prev_j"])
    assert abs(got["electric_j"] - want["electric_j"]) <= 1e-12 * want["electric_j"]


def test_energy_lossless_closed_box_is_bounded():
    """The audit's use: a PEC box with a lossless dielectric, excited then
    left alone, keeps its modified energy constant to round-off
    (audit_periodic_energy.c's invariant) while the raw energy oscillates."""
    from oracle import Scene
    from tests.cases import DT1

    s = Scene(nx=24, ny=20, nz=18, n_steps=120, boxes=[(6, 14, 5, 12, 4, 10, 4.0, 0.0)],
              sources=[(12, 10, 9, 2, 0, 1.0, 0, 10 * DT1, 3 * DT1, 0.0)], probes=[(12, 10, 9, 2)])
    sim = _sim(s, rb.FP64, rb.FUSED)
    mods = []
    try:
        for _ in range(s.n_steps):
            sim.advance(1)
            mods.append(sim.energy()["modified_prev_j"])
    finally:
        sim.close()
    tail = np.array(mods[80:])  # source envelope over (t0 + 6 tau = 28 steps)
    assert np.all(np.isfinite(tail)) and tail.max() > 0
    assert (tail.max() - tail.min()) <= 1e-9 * tail.max()
