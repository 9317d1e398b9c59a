"""Every sweep variant the autotuner may pick (cp.async-fed, TMA-fed
interior, and the persistent work-queue sweeps that take interior and slab
tiles by TMA; each tile height and ring depth): FP64 probe series bit-equal
to the CPU oracle, on scenes large enough to have interior work items and,
for the work-queue sweeps, on every small boundary case of tests/cases.py
(PEC walls with sources on the padded planes, periodic wraps, tensors,
per-component overrides).

The sweep variant is forced per session with RFSYN_FDTD_PLAN
("rows,ring,seg_interior,seg_edge,mode"); the session's info confirms that
the sweep ran with that variant and had work."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle import Scene
from rfsyn_b200 import scenes
from tests.cases import CASES, DT1, scene_run_config, workload_to_scene

pytestmark = pytest.mark.gpu

# (rows per tile, ring depth, mode) of every compiled variant; mode 0
# cp.async interior, 1 TMA interior, 2 work-queue sweeps, 3 work-queue
# sweeps with tile origins shifted to the slab edges, 4 work-queue sweeps
# with narrow (2 tj x 16) tiles over the z slabs (no periodic y / z); a
# fourth value 1 puts every item of modes 2-4 in one queue (one launch); a
# fifth value 3 or 4 gives the interior tiles of modes 2, 3 to the sweep
# whose threads own two rows (FP32; that value is its ring depth)
VARIANTS = {
    rb.FP64: [(8, 3, 2), (8, 4, 2), (8, 3, 3), (8, 4, 3), (8, 3, 4), (8, 4, 4), (8, 4, 2, 1), (8, 3, 4, 1),
              (8, 3, 1), (8, 4, 1), (8, 4, 0), (16, 2, 0)],
    rb.FP32: [(8, 4, 2), (8, 3, 2), (16, 3, 2), (8, 4, 3), (16, 3, 3), (8, 4, 4), (8, 3, 4), (16, 3, 4),
              (8, 4, 2, 1), (8, 4, 4, 1), (16, 3, 4, 1), (8, 4, 1), (8, 3, 1), (16, 3, 1), (8, 6, 0), (8, 5, 0),
              (8, 4, 2, 0, 3), (8, 4, 2, 0, 4), (8, 3, 3, 0, 3), (16, 4, 0), (16, 3, 0)],
}
QUEUE = [v for v in VARIANTS[rb.FP64] if v[2] >= 2]
MODE = {0: "cpasync", 1: "tma", 2: "queue", 3: "queue_shifted", 4: "queue_narrow"}


def _vid(v):
    return "tj%d_ns%d_%s%s%s" % (v[0], v[1], MODE[v[2]], "_single" if len(v) > 3 and v[3] else "",
                                 "_tworows%d" % v[4] if len(v) > 4 and v[4] else "")

SCENES = {
    # the headline recipe at 104^3 (5-cell CPML): interior tiles at k0 = 32, 64
    "c2_104": workload_to_scene(scenes.scaled(scenes.c2(), 104, 120)),
    # periodic y and z (the halo of the end tiles would wrap), CPML on x
    "periodic_yz_cpml_x": Scene(
        nx=24, ny=41, nz=100, n_steps=80, periodic=6, npml=4,
        boxes=[(6, 18, 10, 30, 40, 80, 4.0, 0.01)],
        comps=[(2, 12, 20, 50, 7.0, 0.0), (0, 12, 20, 70, 3.0, 0.02)],
        sources=[(12, 20, 60, 2, 0, 1.0, 0, 20 * DT1, 5 * DT1, 0.0)],
        probes=[(14, 22, 62, 2), (12, 0, 3, 0), (8, 30, 45, 1)], freqs=[30e9]),
    # fully periodic: interior items start at plane 0 and wrap to nx-1
    "periodic_all": Scene(
        nx=18, ny=41, nz=100, n_steps=60, periodic=7,
        boxes=[(3, 12, 10, 25, 35, 70, 2.5, 0.0)],
        sources=[(9, 15, 50, 1, 0, 1.0, 0, 15 * DT1, 4 * DT1, 0.0)],
        probes=[(0, 15, 50, 1), (17, 10, 40, 2), (9, 29, 99, 0)]),
}


@pytest.fixture(scope="module")
def wants():
    return {name: oracle.run_oracle(s) for name, s in SCENES.items()}


def _run(s: Scene, precision: int, variant, monkeypatch, need_interior=True):
    tj, ns, tma = variant[:3]
    uni = variant[3] if len(variant) > 3 else 0
    i2 = variant[4] if len(variant) > 4 else 0
    monkeypatch.setenv("RFSYN_FDTD_PLAN", f"{tj},{ns},32,16,{tma},{uni},{i2}")
    rc = scene_run_config(s, precision, rb.FUSED)
    cs = s.to_c()
    needs_setup = bool(s.boxes or s.comps or s.tensors or s.disp or s.spheres or s.tensor3)
    sim = rb.Sim(rc, oracle.device_setup() if needs_setup else None,
                 C.cast(C.pointer(cs), C.c_void_p) if needs_setup else None)
    try:
        info = sim.info()
        assert (info.tile_j, info.ring_depth, info.tma, info.unified, info.interior_ring2) == (tj, ns, tma, uni, i2)
        assert info.edge_items > 0
        if need_interior and not uni:
            assert info.interior_items > 0
        sim.advance(s.n_steps)
        return sim.probes(), sim.dft()
    finally:
        sim.close()


def _narrow_on_wrap(s: Scene, variant, monkeypatch) -> bool:
    """Mode 4 on a scene with periodic y or z: the session must refuse it."""
    if variant[2] != 4 or not (s.periodic & 6):
        return False
    monkeypatch.setenv("RFSYN_FDTD_PLAN", f"{variant[0]},{variant[1]},32,16,4,{variant[3] if len(variant) > 3 else 0}")
    with pytest.raises(RuntimeError, match="non-periodic y and z"):
        rb.Sim(scene_run_config(s, rb.FP64, rb.FUSED))
    return True


@pytest.mark.parametrize("variant", VARIANTS[rb.FP64], ids=_vid)
@pytest.mark.parametrize("name", list(SCENES))
def test_interior_variant_fp64_bit_exact(wants, name, variant, monkeypatch):
    if _narrow_on_wrap(SCENES[name], variant, monkeypatch):
        return
    td, _ = _run(SCENES[name], rb.FP64, variant, monkeypatch)
    assert np.array_equal(td, wants[name]["td"])


@pytest.mark.parametrize("variant", VARIANTS[rb.FP32], ids=_vid)
def test_interior_variants_fp32_agree(wants, variant, monkeypatch):
    """All FP32 variants evaluate the same expressions in the same order:
    identical probe series; and within the FP32 bound of the FP64 oracle."""
    s = SCENES["c2_104"]
    td, _ = _run(s, rb.FP32, variant, monkeypatch)
    ref, _ = _run(s, rb.FP32, VARIANTS[rb.FP32][-1], monkeypatch)
    assert np.array_equal(td, ref)
    want = wants["c2_104"]["td"]
    err = np.linalg.norm(td - want) / np.linalg.norm(want)
    assert err < 1e-3, err


@pytest.mark.parametrize("variant", QUEUE, ids=_vid)
@pytest.mark.parametrize("name", list(CASES))
def test_queue_sweep_boundary_cases_fp64_bit_exact(name, variant, monkeypatch):
    s = CASES[name]
    if _narrow_on_wrap(s, variant, monkeypatch):
        return
    want = oracle.run_oracle(s)
    td, dft = _run(s, rb.FP64, variant, monkeypatch, need_interior=False)
    assert np.array_equal(td, want["td"])


def test_two_rows_interior_is_fp32_only(monkeypatch):
    monkeypatch.setenv("RFSYN_FDTD_PLAN", "8,4,32,16,2,0,4")
    with pytest.raises(RuntimeError, match="two-rows interior"):
        rb.Sim(scene_run_config(SCENES["c2_104"], rb.FP64, rb.FUSED))


def test_plan_override_rejects_unknown_variant(monkeypatch):
    monkeypatch.setenv("RFSYN_FDTD_PLAN", "12,7,32,16,1")
    s = SCENES["periodic_all"]
    with pytest.raises(RuntimeError, match="names no sweep variant"):
        rb.Sim(scene_run_config(s, rb.FP64, rb.FUSED))
