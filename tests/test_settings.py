"""The config surface (rfsyn_b200.settings, fdtd_b200_apply_setting).

CPU, against rfsyn itself (cli/config.c, cJSON.c, settings.c and presets.c
compiled from its sources into oracle/_ref): config.json files with every
kind of value rfsyn's typed getters meet (numbers, integral and not,
out-of-range longs, strings, booleans, nulls, arrays, missing sections,
duplicate keys) give the same getter results and, through rfsyn's own
settings_build_chain, the same fdtd_sim_config_t and AWGN stage parameters
for several example indices.  Then the GPU section's process-wide settings
(set, read back, refused values leave the setting unchanged, "default"
restores the environment's choice) and the per-run options and per-example
scenes.
GPU: examples run one at a time and as a batch give the same I/Q; without
noise the FP64 chain output is rfsyn's fdtd_simulate_echo series cast to
float, exactly."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import settings

REF_LIB = Path(oracle.__file__).resolve().parent / "_ref" / "librfsyn_ref.so"
needs_ref = pytest.mark.skipif(not REF_LIB.exists(), reason="rfsyn not compiled into oracle/_ref")
SIM_FIELDS = [n for n, _ in rb.FdtdSimConfig._fields_]


class _Transform(C.Structure):
    _fields_ = [("apply", C.c_void_p), ("destroy", C.c_void_p), ("ctx", C.c_void_p)]


class _AwgnCtx(C.Structure):  # awgn_ctx_t (engine/noise/awgn.c:11-14)
    _fields_ = [("snr_db", C.c_float), ("state", C.c_uint64), ("inc", C.c_uint64)]


class _Rng(C.Structure):
    _fields_ = [("state", C.c_uint64), ("inc", C.c_uint64)]


def _ref():
    ref = C.CDLL(str(REF_LIB))
    ref.config_load.restype = C.c_void_p
    ref.config_load.argtypes = [C.c_char_p]
    ref.config_destroy.argtypes = [C.c_void_p]
    ref.config_get.restype = C.c_char_p
    ref.config_get.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
    ref.config_get_double.restype = C.c_double
    ref.config_get_double.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double]
    ref.config_get_long.restype = C.c_long
    ref.config_get_long.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_long]
    ref.config_get_bool.restype = C.c_int
    ref.config_get_bool.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int]
    ref.settings_build_chain.restype = C.c_int
    ref.settings_build_chain.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(_Transform), C.c_size_t,
                                         C.POINTER(C.c_size_t)]
    ref.rng_seed.argtypes = [C.POINTER(_Rng), C.c_uint64, C.c_uint64]
    return ref


CONFIGS = [
    {},
    {"fdtd": {}},
    {"fdtd": {"nx": 64, "ny": 48, "nz": 40, "dx": 5e-4, "courant": 0.9, "n_steps": 300, "npml": 6,
              "t0": 30.0, "tau": 6.5, "src_i": 10, "src_j": 11, "src_k": 12, "probe_i": 20, "probe_j": 21,
              "probe_k": 22},
     "awgn": {"enabled": True, "snr_db": 7.3, "seed": 123456789}},
    {"fdtd": {"nx": 64.5, "ny": "48", "nz": True, "dx": "1e-3", "n_steps": 1e30, "npml": None,
              "src_i": -1, "src_j": -7, "src_k": 3.0, "probe_i": -1, "probe_j": 2.5, "probe_k": -2},
     "awgn": {"enabled": 1, "snr_db": "high", "seed": -5}},
    {"fdtd": {"nx": 9.2233720368547758e18, "ny": -9.2233720368547758e18, "nz": 7},
     "awgn": {"enabled": False}},
    {"fdtd": {"courant": float("nan")}},                 # written as NaN: not JSON
    {"fdtd": {"enabled": False, "nx": 10}},
    {"fdtd": [1, 2, 3], "awgn": "on"},
    {"fdtd": {"nx": 1e-300, "ny": 3, "nz": 2, "src_i": 1e15, "probe_k": -0.0, "gpu.precision": "fp32"}},
]
RAW = [
    # duplicate keys: the first one counts, as cJSON finds it
    '{"fdtd": {"nx": 30, "nx": 40, "t0": 1.5, "t0": 9}, "fdtd": {"ny": 99}}',
    # integers beyond double precision, exponents, negative zero
    '{"fdtd": {"nx": 9007199254740993, "ny": 1E2, "nz": -0, "dx": 2.5e-3, "tau": -0.0}}',
    # literals beyond the double range
    '{"fdtd": {"dx": 1' + '0' * 400 + ', "t0": -1' + '0' * 400 + ', "tau": 1e400, "nx": 1' + '0' * 30 + '}}',
]
KEYS = [("fdtd", k) for k in ("nx", "ny", "nz", "dx", "courant", "n_steps", "npml", "src_i", "src_j", "src_k",
                              "probe_i", "probe_j", "probe_k", "t0", "tau", "enabled", "gpu.precision")] + \
       [("awgn", k) for k in ("enabled", "snr_db", "seed")] + [("nosuch", "nx")]


def _files(tmp_path):
    out = []
    for q, c in enumerate(CONFIGS):
        p = tmp_path / f"c{q}.json"
        p.write_text(json.dumps(c, allow_nan=True))
        out.append(p)
    for q, t in enumerate(RAW):
        p = tmp_path / f"r{q}.json"
        p.write_text(t)
        out.append(p)
    return out


@needs_ref
def test_getters_equal_rfsyn(tmp_path):
    ref = _ref()
    for p in _files(tmp_path):
        rc = ref.config_load(str(p).encode())
        if not rc:                         # text rfsyn's parser refuses
            with pytest.raises(ValueError):
                settings.load(p)
            continue
        mine = settings.load(p)
        try:
            for sec, key in KEYS:
                s, k = sec.encode(), key.encode()
                assert settings.get_long(mine, sec, key, -77) == ref.config_get_long(rc, s, k, -77), (p, key)
                d_ref, d_mine = ref.config_get_double(rc, s, k, -0.25), settings.get_double(mine, sec, key, -0.25)
                assert d_mine == d_ref or (np.isnan(d_mine) and np.isnan(d_ref)), (p, key)
                assert settings.get_bool(mine, sec, key, 7) == ref.config_get_bool(rc, s, k, 7), (p, key)
                g = ref.config_get(rc, s, k)
                assert settings.get(mine, sec, key) == (g.decode() if g is not None else None), (p, key)
        finally:
            ref.config_destroy(rc)


@needs_ref
def test_lenient_number_literals_are_refused_loudly(tmp_path):
    # cJSON reads these through strtod; strict JSON (and this module) refuses
    ref = _ref()
    for q, lit in enumerate(["007", "5.", "-.5"]):
        p = tmp_path / f"lenient{q}.json"
        p.write_text('{"fdtd": {"nx": %s}}' % lit)
        rc = ref.config_load(str(p).encode())
        assert rc
        ref.config_destroy(rc)
        with pytest.raises(ValueError):
            settings.load(p)


@needs_ref
def test_stage_config_equals_rfsyn_chain(tmp_path):
    ref = _ref()
    destroy = C.CFUNCTYPE(None, C.c_void_p)
    for p in _files(tmp_path):
        rc = ref.config_load(str(p).encode())
        if not rc:
            continue
        mine = settings.load(p)
        try:
            for example in (0, 1, 17):
                stages = (_Transform * 4)()
                n = C.c_size_t(0)
                assert ref.settings_build_chain(rc, example, stages, 4, C.byref(n)) == 0
                q = 0
                if settings.get_bool(mine, "fdtd", "enabled", 1):
                    want = C.cast(stages[0].ctx, C.POINTER(rb.FdtdSimConfig)).contents
                    got = settings.build_fdtd_config(mine)
                    for f in SIM_FIELDS:
                        assert getattr(got, f) == getattr(want, f), (p, f)
                    q = 1
                noise = settings.awgn_of(mine, example)
                assert (noise is not None) == (n.value == q + 1), p
                if noise is not None:
                    a = C.cast(stages[q].ctx, C.POINTER(_AwgnCtx)).contents
                    rng = _Rng()
                    ref.rng_seed(C.byref(rng), noise[1], noise[2])
                    assert np.float32(noise[0]) == np.float32(a.snr_db)
                    assert (rng.state, rng.inc) == (a.state, a.inc)
                for s in range(n.value):
                    destroy(stages[s].destroy)(stages[s].ctx)
        finally:
            ref.config_destroy(rc)


@pytest.fixture
def restore_settings():
    yield
    for k in settings.PROCESS_KEYS:
        settings.apply_setting(k, "default")


def test_process_settings_round_trip(restore_settings, monkeypatch):
    monkeypatch.delenv("RFSYN_FDTD_PLAN", raising=False)
    monkeypatch.delenv("RFSYN_FDTD_TUNE", raising=False)
    settings.apply_setting("fdtd.gpu.precision", "fp32")
    assert settings.get_setting("precision") == "fp32"
    settings.apply_setting("gpu.schedule", "split")
    assert settings.get_setting("fdtd.gpu.schedule") == "split"
    settings.apply_setting("plan", "8,4,32,16,4,1")
    assert settings.get_setting("plan") == "8,4,32,16,4,1"
    settings.apply_setting("plan", "auto")
    assert settings.get_setting("plan") == "auto"
    settings.apply_setting("tune", "false")
    assert settings.get_setting("tune") == "false"
    settings.apply_setting("trace", "0")
    assert settings.get_setting("trace") == "false"
    # refused values name the setting and leave it unchanged
    for key, bad in [("precision", "fp16"), ("schedule", "fast"), ("plan", "8,4"), ("plan", "8,4,32,16,4,1,0,0"),
                     ("plan", "8,-4,32,16"), ("plan", "8,4,32,16,"), ("plan", "a,b,c,d"), ("tune", "yes"),
                     ("trace", "")]:
        before = settings.get_setting(key)
        with pytest.raises(ValueError, match=key):
            settings.apply_setting(key, bad)
        assert settings.get_setting(key) == before
    with pytest.raises(ValueError, match="unknown setting"):
        settings.apply_setting("gpu.colour", "red")
    # "default" hands the choice back to the environment
    monkeypatch.setenv("RFSYN_FDTD_PLAN", "16,3,32,16,2")
    settings.apply_setting("plan", "default")
    assert settings.get_setting("plan") == "16,3,32,16,2"
    monkeypatch.setenv("RFSYN_FDTD_TUNE", "0")
    settings.apply_setting("tune", "default")
    assert settings.get_setting("tune") == "false"


def test_config_file_applies_gpu_section(restore_settings):
    cfg = {"fdtd": {"gpu.precision": "fp32", "gpu.schedule": "split", "gpu.tune": 0, "gpu.trace": False,
                    "gpu.batch": 4}}
    settings.apply_gpu_settings(cfg)
    assert settings.get_setting("precision") == "fp32" and settings.get_setting("schedule") == "split"
    assert settings.get_setting("tune") == "false" and settings.get_setting("trace") == "false"
    with pytest.raises(ValueError, match="unknown setting fdtd.gpu.precission"):
        settings.apply_gpu_settings({"fdtd": {"gpu.precission": "fp32"}})
    with pytest.raises(ValueError, match="gpu.schedule"):
        settings.apply_gpu_settings({"fdtd": {"gpu.schedule": 3}})


def test_run_options():
    o = settings.run_options({"fdtd": {"gpu.batch": 8, "gpu.dft_bins": 5, "gpu.dft_f_lo_hz": 1e9,
                                       "gpu.dft_f_hi_hz": 3e9, "gpu.scene_seed": 9}})
    assert (o.batch, o.dft_bins, o.scene_seed) == (8, 5, 9)
    assert o.freqs() == list(np.linspace(1e9, 3e9, 5))
    assert settings.run_options({}) == settings.RunOptions()
    for bad in [{"gpu.batch": 0}, {"gpu.batch": 2.5}, {"gpu.batch": "4"}, {"gpu.dft_bins": -1},
                {"gpu.dft_f_lo_hz": float("inf")}, {"gpu.scene_seed": True},
                {"gpu.dft_bins": 3, "gpu.dft_f_lo_hz": 5e9, "gpu.dft_f_hi_hz": 1e9}]:
        with pytest.raises(ValueError):
            settings.run_options({"fdtd": bad})


def test_example_workloads(restore_settings):
    base = {"fdtd": {"nx": 40, "ny": 36, "nz": 44, "n_steps": 80, "t0": 20.0, "tau": 5.0}}
    w0 = settings.example_workload(base, 0)
    w5 = settings.example_workload(base, 5)
    # without a scene seed every example simulates the same empty grid, as rfsyn does
    assert w0.boxes == w5.boxes == [] and w0.spheres == w5.spheres == []
    s = settings.build_fdtd_config(base)
    src = w0.sources[0]
    assert (src["i"], src["j"], src["k"]) == (s.src_i, s.src_j, s.src_k) == (20, 18, 22)
    assert (w0.probes[0]["i"], w0.probes[0]["j"], w0.probes[0]["k"]) == (26, 18, 22)
    dt = rb.dt_of(1e-3, 0.99)
    assert src["p0"] == 20.0 * dt and src["p1"] == 5.0 * dt and src["waveform"] == rb.WAVE_GAUSSIAN_DERIV
    seeded = {"fdtd": dict(base["fdtd"], **{"gpu.scene_seed": 3})}
    a = [settings.example_workload(seeded, i) for i in range(6)]
    b = [settings.example_workload(seeded, i) for i in range(6)]
    assert [(w.boxes, w.spheres) for w in a] == [(w.boxes, w.spheres) for w in b]
    assert len({repr((w.boxes, w.spheres)) for w in a}) > 3          # examples differ
    assert any(w.boxes or w.spheres for w in a)
    settings.apply_setting("precision", "fp32")
    assert settings.example_workload(base, 0).precision == rb.FP32
    for bad in [{"n_steps": 0}, {"src_i": 41}, {"probe_k": 45}, {"nx": 0}, {"dx": -1e-3}]:
        with pytest.raises(ValueError):
            settings.example_workload({"fdtd": dict(base["fdtd"], **bad)}, 0)
    with pytest.raises(ValueError, match="scene_seed"):
        settings.example_workload({"fdtd": {"nx": 20, "gpu.scene_seed": 1}}, 0)


@pytest.mark.gpu
@needs_ref
def test_examples_batched_equal_single_and_rfsyn(restore_settings, tmp_path):
    ref = _ref()
    ref.fdtd_simulate_echo.argtypes = [C.POINTER(rb.FdtdSimConfig), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    base = {"fdtd": {"nx": 32, "ny": 30, "nz": 34, "n_steps": 120, "npml": 6, "t0": 24.0, "tau": 6.0,
                     "gpu.precision": "fp64"},
            "awgn": {"enabled": False}}
    one = settings.run_examples(base, range(3))
    # without noise the chain's output is rfsyn's FP64 series cast to float, imaginary part 0
    s = settings.build_fdtd_config(base)
    td = np.zeros(s.n_steps)
    fs = C.c_double()
    assert ref.fdtd_simulate_echo(C.byref(s), td.ctypes.data_as(C.POINTER(C.c_double)), C.byref(fs)) == 0
    for iq in one:
        assert np.array_equal(iq.real, td.astype(np.float32)) and not iq.imag.any()
    # seeded scenes with noise: batched equals one at a time, examples differ
    seeded = {"fdtd": dict(base["fdtd"], **{"gpu.scene_seed": 5, "gpu.precision": "fp32"}),
              "awgn": {"enabled": True, "snr_db": 10.0, "seed": 77}}
    single = settings.run_examples(seeded, range(4))
    batched = settings.run_examples({"fdtd": dict(seeded["fdtd"], **{"gpu.batch": 4}), "awgn": seeded["awgn"]},
                                    range(4))
    for x, y in zip(single, batched):
        assert np.array_equal(x, y)
    assert not np.array_equal(single[0], single[1])
    paths = settings.write_examples(seeded, [2], tmp_path)
    assert Path(paths[0]).name == "example_000002.iq"
    assert np.array_equal(np.fromfile(paths[0], dtype=np.complex64), single[2])


def test_setting_text_and_disabled_stage():
    assert settings.setting_text(True) == "true" and settings.setting_text(False) == "false"
    assert settings.setting_text(0) == "0" and settings.setting_text(4.0) == "4"
    assert settings.setting_text(2.5) == "2.5" and settings.setting_text("8,4,128,32,2") == "8,4,128,32,2"
    with pytest.raises(ValueError):
        settings.setting_text(None)
    with pytest.raises(ValueError, match="fdtd.enabled"):
        settings.run_examples({"fdtd": {"enabled": False}}, [0])
    # the AWGN stage of example i: (float) snr, seed as uint64, stream i
    assert settings.awgn_of({"awgn": {"snr_db": 7.3, "seed": -1}}, 5) == (float(np.float32(7.3)), (1 << 64) - 1, 5)
    assert settings.awgn_of({"awgn": {"enabled": False}}, 0) is None
