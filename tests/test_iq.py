"""The FDTD stage's output signal with rfsyn's AWGN, computed on the GPU
(fdtd_b200_sim_read_iq), and the .iq writer (fdtd_b200_iq_write).

CPU: the generator jump-ahead the kernel uses (PCG32 stepped d times as one
affine map) equals rfsyn's own PCG32 stepped one by one (engine/core/rng.c,
compiled from its sources into oracle/_ref); the .iq writer stores
interleaved float32 I/Q as rfsyn's write_signal does.
GPU: without noise the signal is (float) of the probe series exactly; with
noise it equals rfsyn's awgn_create(...).apply on the same signal: the same
uniforms (integer arithmetic, exact), the same noise scale (the power summed
in rfsyn's order), and the Box-Muller pair with logf / cosf / sinf taken as
the rounding of double-precision values (the correctly rounded float in
all but rare ties).  glibc's logf / cosf / sinf are accurate to under one
ulp but not always correctly rounded, so a few per cent of the samples
differ in the last bit; the bar is 2 ulps of the larger of the sample and
its noise term everywhere, and 95 % of the samples bit-identical (97.6 %
measured on B200)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle import Scene
from tests.cases import DT1, scene_run_config

REF_LIB = Path(oracle.__file__).resolve().parent / "_ref" / "librfsyn_ref.so"
MASK = (1 << 64) - 1
MULT = 6364136223846793005
needs_ref = pytest.mark.skipif(not REF_LIB.exists(), reason="rfsyn not compiled into oracle/_ref")


class _Rng(C.Structure):
    _fields_ = [("state", C.c_uint64), ("inc", C.c_uint64)]


class _Signal(C.Structure):  # the leading fields of rfsyn's signal_t
    _fields_ = [("samples", C.POINTER(C.c_float)), ("n_samples", C.c_size_t)]


class _Transform(C.Structure):
    _fields_ = [("apply", C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p)), ("destroy", C.c_void_p),
                ("ctx", C.c_void_p)]


def _ref():
    ref = C.CDLL(str(REF_LIB))
    ref.rng_seed.argtypes = [C.POINTER(_Rng), C.c_uint64, C.c_uint64]
    ref.rng_next_u32.restype = C.c_uint32
    ref.rng_next_u32.argtypes = [C.POINTER(_Rng)]
    ref.signal_create.restype = C.POINTER(_Signal)
    ref.signal_create.argtypes = [C.c_size_t, C.c_double, C.c_double]
    ref.signal_destroy.argtypes = [C.POINTER(_Signal)]
    ref.awgn_create.restype = _Transform
    ref.awgn_create.argtypes = [C.c_float, C.c_uint64, C.c_uint64]
    return ref


def pcg32_advance(state: int, inc: int, delta: int) -> int:
    """x -> MULT x + inc applied delta times, composed by squaring."""
    acc_mult, acc_plus, cur_mult, cur_plus = 1, 0, MULT, inc
    while delta:
        if delta & 1:
            acc_mult = (acc_mult * cur_mult) & MASK
            acc_plus = (acc_plus * cur_mult + cur_plus) & MASK
        cur_plus = ((cur_mult + 1) * cur_plus) & MASK
        cur_mult = (cur_mult * cur_mult) & MASK
        delta >>= 1
    return (acc_mult * state + acc_plus) & MASK


@needs_ref
@pytest.mark.parametrize("seed,stream", [(7, 0), (123456789, 5), (2**63 + 11, 2**40)])
def test_jump_ahead_equals_rfsyn_sequential_pcg32(seed, stream):
    ref = _ref()
    g = _Rng()
    ref.rng_seed(C.byref(g), seed, stream)
    start, inc = g.state, g.inc
    for delta in (0, 1, 2, 3, 17, 1000, 4095):
        h = _Rng(start, inc)
        for _ in range(delta):
            ref.rng_next_u32(C.byref(h))
        assert pcg32_advance(start, inc, delta) == h.state


def test_iq_write_stores_interleaved_float32(tmp_path):
    lib = rb.load()
    iq = (np.arange(10, dtype=np.float32) * 0.5 - 1.0)
    p = tmp_path / "sig.iq"
    assert lib.fdtd_b200_iq_write(str(p).encode(), iq.ctypes.data_as(C.POINTER(C.c_float)), 5) == 0
    assert p.read_bytes() == iq.tobytes()
    q = tmp_path / "empty.iq"
    assert lib.fdtd_b200_iq_write(str(q).encode(), None, 0) == 0 and q.read_bytes() == b""
    assert lib.fdtd_b200_iq_write(None, iq.ctypes.data_as(C.POINTER(C.c_float)), 5) == -1
    assert lib.fdtd_b200_iq_write(str(tmp_path / "no" / "dir.iq").encode(),
                                  iq.ctypes.data_as(C.POINTER(C.c_float)), 5) == -1


# ---------------------------------------------------------------- GPU --------
def _scene(n_steps=700):
    return Scene(nx=20, ny=18, nz=16, n_steps=n_steps, npml=4,
                 sources=[(10, 9, 8, 2, 0, 1.0, 2, 30e9, 60 * DT1, 15 * DT1)],
                 probes=[(13, 9, 8, 2), (7, 11, 6, 0)])


def _rfsyn_awgn(ref, x: np.ndarray, snr_db: float, seed: int, stream: int) -> np.ndarray:
    sig = ref.signal_create(x.size, 1e9, 0.0)
    buf = np.ctypeslib.as_array(sig.contents.samples, shape=(2 * x.size,))
    buf[0::2] = x.astype(np.float32)
    buf[1::2] = 0.0
    t = ref.awgn_create(snr_db, seed, stream)
    assert t.apply(t.ctx, C.cast(sig, C.c_void_p)) == 0
    out = buf.copy().view(np.complex64)
    C.CFUNCTYPE(None, C.c_void_p)(t.destroy)(t.ctx)
    ref.signal_destroy(sig)
    return out


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("precision", [rb.FP64, rb.FP32], ids=["fp64", "fp32"])
def test_device_iq_equals_rfsyn_chain(precision):
    ref = _ref()
    s = _scene()
    sim = rb.Sim(scene_run_config(s, precision, rb.FUSED))
    try:
        sim.advance(s.n_steps)
        td = sim.probes()
        for p in range(2):
            clean = sim.read_iq(p)
            assert np.array_equal(clean.real, td[p].astype(np.float32))
            assert np.all(clean.imag == 0.0)
            for snr, seed, stream in ((10.0, 42, 0), (-3.0, 2**40 + 7, 9)):
                got = sim.read_iq(p, snr, seed, stream)
                want = _rfsyn_awgn(ref, td[p], snr, seed, stream)
                assert np.abs(want - clean).max() > 0          # noise was added
                noise = want - clean
                for part, w, nz in ((got.real, want.real, noise.real), (got.imag, want.imag, noise.imag)):
                    # 2 ulps of the larger of the sample and its noise term
                    scale = np.maximum(np.abs(w), np.abs(nz)).astype(np.float32)
                    assert np.all(np.abs(part - w) <= 2 * np.spacing(scale))
                    assert np.mean(part == w) >= 0.95
    finally:
        sim.close()


@pytest.mark.gpu
def test_batch_scene_iq_equals_single_scene():
    from rfsyn_b200 import scenes

    ws = scenes.c4(seed=11, n_scenes=3, precision=rb.FP32, n_steps=120, lo=20, hi=40, npml=4)
    setups = [scenes.scene_setup(w) for w in ws]
    b = rb.Batch([scenes.run_config(w) for w in ws], [s.ptr if s else None for s in setups])
    try:
        b.advance(ws[0].n_steps)
        b.synchronize()
        for q, w in enumerate(ws):
            sim = rb.Sim(scenes.run_config(w), setups[q].ptr if setups[q] else None)
            try:
                sim.advance(w.n_steps)
                for p in (0, 3):
                    assert np.array_equal(b.read_iq(q, p, 6.0, 9, q), sim.read_iq(p, 6.0, 9, q))
                    assert np.array_equal(b.read_iq(q, p), sim.read_iq(p))
            finally:
                sim.close()
    finally:
        b.close()
