"""The periodic-cell recipe (rfsyn_b200.scenes.c3: TF/SF plane wave, tilted
slab of a full 3x3 eps_r, 2-pole Lorentz layer, reflection / transmission
probe planes) at a size the oracle runs in seconds: FP64 device runs equal
the CPU oracle bit for bit, through the oracle's explicit samples and
through the product's own slab / dispersive-box helpers alike; FP32 probe
spectra within 1e-4 relative L2 of the FP64 oracle, probe by probe."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import scenes
from tests.cases import run_device, workload_to_scene

FP32_SPEC_L2 = 1e-4


def _workload(precision):
    return scenes.c3(seed=7, precision=precision, nx=12, ny=10, nz=96, n_steps=260, npml=6, grid_probes=2)


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
    assert np.array_equal(r["td"], want["td"])


@pytest.mark.gpu
def test_fp32_spectra_within_bound(want):
    w = _workload(rb.FP32)
    st = scenes.scene_setup(w)
    r = rb.run(scenes.run_config(w), st.ptr, None)
    # each probe against its own FP64 norm (no normalisation by the largest)
    err = np.linalg.norm(r["dft"] - want["dft"], axis=1) / np.linalg.norm(want["dft"], axis=1)
    assert err.max() <= FP32_SPEC_L2, (int(err.argmax()), float(err.max()))
