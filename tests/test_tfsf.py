"""Plane-wave injection through a total-field / scattered-field boundary (no
rfsyn counterpart).

CPU (oracle), the physics that pins the restatement:
  * normal incidence on a closed box in vacuum: outside the box the field
    stays at rounding level (the line and the grid propagate identically);
    inside, the probe sees the incident pulse;
  * oblique incidence (several directions, mixed polarisations): leakage
    into the scattered region below -60 dB of the incident peak for a pulse
    whose spectrum is 20 dB down at 17 cells per wavelength, below -55 dB at
    9 cells per wavelength (the dispersion-matched line); along the body
    diagonal the line reproduces the grid exactly;
  * normal incidence on a dielectric half-space (periodic x / y, eps_r 4):
    the reflected pulse in the scattered region is -1/3 of the incident one.
GPU: FP64 device runs equal the oracle bit for bit (box with CPML, oblique;
periodic x / y with a slab; both schedules); FP32 within the FP32 bound."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle import Scene
from tests.cases import DT1, run_device

GD = dict(waveform=0, p0=40 * DT1, p1=10 * DT1, p2=0.0)


def box_scene(theta=0.0, phi=0.0, psi=0.0, n_steps=160, tau=10):
    gd = dict(waveform=0, p0=4 * tau * DT1, p1=tau * DT1, p2=0.0)
    return Scene(nx=36, ny=34, nz=40, n_steps=n_steps, npml=6,
                 plane_wave=dict(theta=theta, phi=phi, psi=psi, amplitude=1.0, i0=12, i1=24, j0=11, j1=23,
                                 k0=12, k1=28, **gd),
                 probes=[(18, 17, 20, 0), (18, 17, 20, 1), (18, 17, 20, 2),      # inside
                         (18, 17, 9, 0), (18, 17, 31, 0), (9, 17, 20, 2),         # outside
                         (27, 17, 20, 1), (18, 8, 20, 0), (18, 26, 20, 2),
                         (10, 9, 10, 0), (26, 25, 30, 1), (10, 25, 10, 2)])     # outside, near corners


def leakage_db(theta, phi, psi, tau):
    td = oracle.run_oracle(box_scene(theta, phi, psi, n_steps=200, tau=tau))["td"]
    peak = np.abs(td[:3]).max()
    assert peak > 0.3
    return 20 * math.log10(np.abs(td[3:]).max() / peak)


def test_normal_incidence_box_has_no_leakage():
    td = oracle.run_oracle(box_scene())["td"]
    peak = np.abs(td[0]).max()
    assert peak > 0.5      # the incident E along x reaches the centre
    assert np.abs(td[1:3]).max() < 1e-12 * peak   # no cross components
    assert np.abs(td[3:]).max() < 1e-12 * peak    # nothing leaks out


OBLIQUE = [(30, 20, 0.6), (45, 45, 0.3), (15, 0, 0.0), (40, -70, 1.2)]


@pytest.mark.parametrize("theta,phi,psi", OBLIQUE, ids=[f"t{a}p{b}" for a, b, _ in OBLIQUE])
def test_oblique_incidence_leakage(theta, phi, psi):
    # tau 20 dt: spectrum 20 dB down at ~17 cells per wavelength; tau 10 dt: ~9
    assert leakage_db(math.radians(theta), math.radians(phi), psi, tau=20) < -60.0
    assert leakage_db(math.radians(theta), math.radians(phi), psi, tau=10) < -55.0


def test_body_diagonal_line_is_exact():
    # along (1,1,1) the grid's dispersion equals the line's at d1 = dx / sqrt 3
    assert leakage_db(math.atan(math.sqrt(2.0)), math.radians(45), 1.0, tau=10) < -150.0


def test_fresnel_half_space_normal_incidence():
    nz, kz0, kint = 400, 60, 200
    s = Scene(nx=4, ny=4, nz=nz, n_steps=900, periodic=3, npml=10,
              plane_wave=dict(theta=0.0, phi=0.0, psi=0.0, amplitude=1.0, i0=0, i1=3, j0=0, j1=3,
                              k0=kz0, k1=nz - 30, waveform=0, p0=80 * DT1, p1=20 * DT1, p2=0.0),
              boxes=[(0, 4, 0, 4, kint, nz - 10, 4.0, 0.0)],
              probes=[(1, 1, kz0 - 10, 0), (1, 1, (kz0 + kint) // 2, 0)])
    td = oracle.run_oracle(s)["td"]
    refl = td[0]
    # incident pulse at the mid probe, before the reflection comes back
    inc = td[1][: 520]
    r = refl[np.argmax(np.abs(refl))] / inc[np.argmax(np.abs(inc))]
    assert abs(r - (-1.0 / 3.0)) < 0.02, r


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [rb.FUSED, rb.SPLIT], ids=["fused", "split"])
def test_device_fp64_box_oblique_equals_oracle(schedule):
    s = box_scene(theta=math.radians(35), phi=math.radians(-25), psi=1.1, n_steps=90)
    want = oracle.run_oracle(s)
    got = run_device(s, rb.FP64, schedule)
    assert np.array_equal(got["td"], want["td"])


@pytest.mark.gpu
def test_device_fp64_periodic_slab_equals_oracle():
    s = Scene(nx=8, ny=6, nz=120, n_steps=220, periodic=3, npml=8,
              plane_wave=dict(theta=0.0, phi=0.0, psi=0.4, amplitude=1.0, i0=0, i1=7, j0=0, j1=5, k0=20, k1=100,
                              **GD),
              boxes=[(0, 8, 0, 6, 50, 70, 3.0, 0.01)],
              probes=[(2, 2, 15, 0), (2, 2, 15, 1), (3, 3, 60, 0), (3, 3, 80, 1), (1, 1, 105, 4)])
    want = oracle.run_oracle(s)
    got = run_device(s, rb.FP64, rb.FUSED)
    assert np.array_equal(got["td"], want["td"])


@pytest.mark.gpu
def test_device_fp32_within_bound():
    s = box_scene(theta=math.radians(30), phi=math.radians(20), psi=0.6, n_steps=120)
    want = oracle.run_oracle(s)["td"]
    got = run_device(s, rb.FP32, rb.FUSED)["td"]
    scale = np.abs(want).max()
    assert np.abs(got - want).max() / scale < 1e-3


def test_oblique_incidence_along_a_periodic_axis_is_rejected():
    # host-side check before any device work (runs without a GPU): a k
    # component along a wrapped axis would need Floquet boundaries
    from tests.cases import scene_run_config

    s = Scene(nx=8, ny=6, nz=60, n_steps=10, periodic=3, npml=8,
              plane_wave=dict(theta=math.radians(20), phi=0.0, psi=0.0, amplitude=1.0, i0=0, i1=7, j0=0, j1=5,
                              k0=20, k1=40, **GD), probes=[(2, 2, 15, 0)])
    with pytest.raises(RuntimeError, match="periodic axis 0"):
        rb.run(scene_run_config(s, rb.FP64, rb.FUSED))
