"""The headline scene recipe (smoothed dielectric spheres, Debye spheres,
CPML, many probes, DFT) at oracle-friendly size: FP64 device runs bit-equal
to the CPU oracle, FP32 probe spectra within the stated relative-L2 bound."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import scenes
from tests.cases import run_device, workload_to_scene

pytestmark = pytest.mark.gpu
FP32_SPEC_L2 = 1e-4


def _scene(n=64, steps=400):
    return workload_to_scene(scenes.scaled(scenes.c2(), n, steps))


@pytest.fixture(scope="module")
def want():
    return oracle.run_oracle(_scene())


@pytest.mark.parametrize("schedule", [rb.SPLIT, rb.FUSED])
def test_scaled_c2_fp64_bit_exact(want, schedule):
    got = run_device(_scene(), rb.FP64, schedule)
    assert np.array_equal(got["td"], want["td"])


def test_scaled_c2_fp32_spectrum(want):
    got = run_device(_scene(), rb.FP32, rb.FUSED)
    errs = [np.linalg.norm(got["dft"][p] - want["dft"][p]) / np.linalg.norm(want["dft"][p])
            for p in range(want["dft"].shape[0])]
    assert max(errs) <= FP32_SPEC_L2, max(errs)
