"""The periodic-cell recipe (rfsyn_b200.scenes.c3: TF/SF plane wave, tilted
slab of a full 3x3 eps_r with subpixel-smoothed faces, 2-pole Lorentz layer,
reflection / transmission probe planes) at a size the oracle runs in
seconds.  The oracle builds the smoothed slab's rows itself
(oracle.subpixel_oracle); the product builds them on the GPU.  FP64 device
runs equal the CPU oracle bit for bit when both run the same rows (the
oracle's explicit samples, or the rows the product's GPU helper built), and
within 1e-12 of the probe peak when each builds its own; the rows themselves
agree to 1e-13; the staircased slab stays bit-exact through the product's
own helpers; FP32 probe spectra within 1e-4 relative L2 of the FP64 oracle,
probe by probe."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import scenes
from tests.cases import oracle_slab_rows, run_device, slab_rows, workload_to_scene

FP32_SPEC_L2 = 1e-4


def _workload(precision, slab_smoothing=1):
    # 900 steps: the whole pulse crosses the transmission plane (with fewer,
    # those probes see only its leading edge, a signal too weak to grade)
    return scenes.c3(seed=7, precision=precision, nx=12, ny=10, nz=96, n_steps=900, npml=6, grid_probes=2,
                     slab_smoothing=slab_smoothing)


def _close(got, want, tol=1e-12):
    scale = np.abs(want).max(axis=1, keepdims=True)
    return float((np.abs(got - want) / scale).max()) <= tol


@pytest.fixture(scope="module")
def want():
    s = workload_to_scene(_workload(rb.FP64))
    assert s.tensor3 and s.disp and s.plane_wave
    return oracle.run_oracle(s)


def test_oracle_sees_the_wave(want):
    td = want["td"]
    assert np.abs(td[:4]).max() > 0      # reflected field below the boundary
    assert np.abs(td[4:]).max() > 0      # transmitted field


@pytest.mark.gpu
def test_fp64_device_equals_oracle(want):
    got = run_device(workload_to_scene(_workload(rb.FP64)), rb.FP64, rb.FUSED)
    assert np.array_equal(got["td"], want["td"])


@pytest.mark.gpu
def test_fp64_product_helpers_equal_oracle(want):
    w = _workload(rb.FP64)
    st = scenes.scene_setup(w)
    r = rb.run(scenes.run_config(w), st.ptr, None)
    # the same rows on both sides: bit for bit
    same = oracle.run_oracle(workload_to_scene(w, slab_source="product"))
    assert np.array_equal(r["td"], same["td"])
    # each side its own rows: within 1e-12 of each probe's peak
    assert _close(r["td"], want["td"])


@pytest.mark.gpu
def test_smoothed_slab_rows_equal_the_oracle_restatement():
    w = _workload(rb.FP64)
    got = {r[:4]: np.array(r[4]) for r in slab_rows(w)}
    want = {r[:4]: np.array(r[4]) for r in oracle_slab_rows(w)}
    assert got.keys() == want.keys()
    assert max(float(np.abs(got[k] - want[k]).max()) for k in got) <= 1e-13
    # the faces carry mixed rows, not eps_r^-1 of the slab
    minv = np.linalg.inv(np.reshape(w.slabs[0][3], (3, 3)))
    mixed = [k for k in got if not np.allclose(got[k], minv[k[0]], rtol=1e-12, atol=0)]
    assert mixed and all(np.all(np.isfinite(got[k])) for k in mixed)


@pytest.mark.gpu
def test_fp64_staircased_slab_product_helpers_equal_oracle():
    w = _workload(rb.FP64, slab_smoothing=0)
    st = scenes.scene_setup(w)
    r = rb.run(scenes.run_config(w), st.ptr, None)
    assert np.array_equal(r["td"], oracle.run_oracle(workload_to_scene(w))["td"])


@pytest.mark.gpu
def test_fp32_spectra_within_bound(want):
    w = _workload(rb.FP32)
    st = scenes.scene_setup(w)
    r = rb.run(scenes.run_config(w), st.ptr, None)
    # each probe against its own FP64 norm (no normalisation by the largest)
    err = np.linalg.norm(r["dft"] - want["dft"], axis=1) / np.linalg.norm(want["dft"], axis=1)
    assert err.max() <= FP32_SPEC_L2, (int(err.argmax()), float(err.max()))
