"""GPU parity: every path through the C ABI against rfsyn's golden outputs
and the CPU oracle.

FP64 runs are required to be bit-for-bit equal to rfsyn for time-domain
samples (the kernels keep rfsyn's operation order and never contract to
FMA); probe DFTs use CUDA's sincos instead of libm and are held to 1e-12
relative.  FP32 runs are held to the probe-spectrum relative L2 bound of
1e-4 against the FP64 result."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from tests.cases import CASES, c1_scene, run_device, simulate_unit_cfg

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
DFT_RTOL = 1e-12      # FP64 DFT (device sincos vs libm)
FP32_SPEC_L2 = 1e-4   # FP32 probe spectrum vs FP64


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("schedule", [rb.SPLIT, rb.FUSED])
@pytest.mark.parametrize("name", sorted(CASES))
def test_device_loop_fp64_bit_exact(name, schedule):
    g = np.load(GOLDEN / f"{name}.npz")
    r = run_device(CASES[name], rb.FP64, schedule)
    assert np.array_equal(r["td"], g["td"]), np.abs(r["td"] - g["td"]).max()
    if g["dft"].size:
        assert rel_l2(r["dft"], g["dft"]) <= DFT_RTOL


@pytest.mark.parametrize("name", sorted(CASES))
def test_stepwise_api_fp64_bit_exact(name):
    # rfsyn's fdtd_update_* called one step at a time on host arrays
    g = np.load(GOLDEN / f"{name}.npz")
    r = oracle.run_stepwise(CASES[name])
    assert np.array_equal(r["td"], g["td"])
    assert np.array_equal(r["dft"], g["dft"])


@pytest.mark.parametrize("mask", range(8))
def test_stepwise_fields_all_periodic_masks(mask):
    # rfsyn tests/periodic_wrapping_unit.c: arbitrary fields on a 5x6x7 grid
    from oracle import Scene

    s = Scene(nx=5, ny=6, nz=7, n_steps=3, periodic=mask, npml=1,
              boxes=[(1, 3, 1, 4, 2, 5, 3.0, 0.02)], comps=[(0, 2, 2, 2, 5.0, 0.0), (2, 1, 3, 3, 2.0, 0.1)])
    ini = np.random.default_rng(7).uniform(-1e-3, 1e-3, size=(6, 6, 7, 8))
    assert np.array_equal(oracle.fields_stepwise(s, ini), oracle.fields_oracle(s, ini))


def test_simulate_echo_matches_rfsyn_unit():
    # rfsyn tests/simulate_unit.c: finite, nonconstant, quiet start,
    # bit-for-bit determinism, and bit-equal to rfsyn's own samples
    g = np.load(GOLDEN / "simulate_unit.npz")
    cfg = simulate_unit_cfg()
    rc_a, a, fs_a = rb.simulate_echo(cfg)
    rc_b, b, fs_b = rb.simulate_echo(cfg)
    assert rc_a == 0 and rc_b == 0
    assert fs_a == fs_b == float(g["fs"])
    assert np.all(np.isfinite(a))
    assert a.tobytes() == b.tobytes()
    peak = np.abs(a).max()
    assert peak > 1e-9 and a.max() - a.min() > 1e-9
    assert np.abs(a[:20]).max() < 1e-3 * peak
    assert np.array_equal(a, g["td"])


@pytest.mark.parametrize("precision", [rb.FP64, rb.FP32])
def test_stage_apply_writes_float_samples(precision):
    lib = rb.load()
    lib.fdtd_b200_set_default_precision(precision)
    try:
        class Signal(C.Structure):
            _fields_ = [("samples", C.c_void_p), ("n_samples", C.c_size_t), ("sample_rate_hz", C.c_double),
                        ("center_freq_hz", C.c_double), ("metadata", C.c_void_p), ("meta_copy", C.c_void_p),
                        ("meta_free", C.c_void_p)]

        class Transform(C.Structure):
            _fields_ = [("apply", C.c_void_p), ("destroy", C.c_void_p), ("ctx", C.c_void_p)]

        lib.fdtd_stage_create.restype = Transform
        lib.fdtd_stage_create.argtypes = [C.c_void_p]
        lib.signal_create.restype = C.POINTER(Signal)
        lib.signal_create.argtypes = [C.c_size_t, C.c_double, C.c_double]
        lib.signal_destroy.argtypes = [C.POINTER(Signal)]
        cfg = simulate_unit_cfg()
        t = lib.fdtd_stage_create(C.byref(cfg))
        sig = lib.signal_create(0, 0.0, 0.0)
        apply = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(Signal))(t.apply)
        assert apply(t.ctx, sig) == 0
        n = sig.contents.n_samples
        assert n == cfg.n_steps
        iq = np.ctypeslib.as_array(C.cast(sig.contents.samples, C.POINTER(C.c_float)), shape=(2 * n,))
        g = np.load(GOLDEN / "simulate_unit.npz")
        assert sig.contents.sample_rate_hz == float(g["fs"])
        assert np.all(iq[1::2] == 0)
        if precision == rb.FP64:
            assert np.array_equal(iq[0::2], g["td"].astype(np.float32))
        else:
            assert rel_l2(iq[0::2].astype(np.float64), g["td"]) < 1e-3
        C.CFUNCTYPE(None, C.c_void_p)(t.destroy)(t.ctx)
        lib.signal_destroy(sig)
    finally:
        lib.fdtd_b200_set_default_precision(rb.FP64)


@pytest.mark.parametrize("schedule", [rb.SPLIT, rb.FUSED])
def test_c1_fp64_against_rfsyn(schedule):
    g = np.load(GOLDEN / "c1.npz")
    r = run_device(c1_scene(), rb.FP64, schedule)
    assert np.array_equal(r["td"], g["td"])
    assert rel_l2(r["dft"], g["dft"]) <= DFT_RTOL


@pytest.mark.parametrize("schedule", [rb.SPLIT, rb.FUSED])
def test_c1_fp32_spectrum_within_bound(schedule):
    g = np.load(GOLDEN / "c1.npz")
    r = run_device(c1_scene(), rb.FP32, schedule)
    for p in range(g["dft"].shape[0]):
        err = rel_l2(r["dft"][p], g["dft"][p])
        assert err <= FP32_SPEC_L2, (p, err)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32_schedules_agree_with_fp64(name):
    g = np.load(GOLDEN / f"{name}.npz")
    a = run_device(CASES[name], rb.FP32, rb.SPLIT)
    b = run_device(CASES[name], rb.FP32, rb.FUSED)
    for p in range(g["td"].shape[0]):
        scale = max(np.abs(g["td"][p]).max(), 1e-30)
        assert np.abs(a["td"][p] - g["td"][p]).max() / scale < 5e-4
        assert np.abs(b["td"][p] - g["td"][p]).max() / scale < 5e-4


def test_session_reset_is_repeatable():
    s = CASES["cpml_materials"]
    from tests.cases import scene_run_config

    rc = scene_run_config(s, rb.FP32, rb.FUSED)
    cs = s.to_c()
    sim = rb.Sim(rc, oracle.device_setup(), C.cast(C.pointer(cs), C.c_void_p))
    sim.advance(s.n_steps)
    a = sim.probes()
    sim.reset()
    sim.advance(17)
    sim.advance(s.n_steps - 17)
    b = sim.probes()
    sim.close()
    assert a.tobytes() == b.tobytes()


def test_extension_rejects_bad_config():
    rc = rb.RunConfig(8, 8, 8, 1e-3, 10, 2, sources=[dict(i=9, j=1, k=1)])
    with pytest.raises(RuntimeError):
        rb.run(rc)
    rc = rb.RunConfig(8, 8, 8, 1e-3, 10, 2, probes=[dict(i=1, j=1, k=1, component=7)])
    with pytest.raises(RuntimeError):
        rb.run(rc)
    rc = rb.RunConfig(8, 8, 8, 1e-3, 10, 4)
    with pytest.raises(RuntimeError):
        rb.run(rc)
