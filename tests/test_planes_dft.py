"""Plane probes and the running DFT.

A plane probe records, every step, the mean of one field component over a
whole grid plane; in a cell periodic across the plane at normal incidence
that is the specular wave, so its spectrum is a reflection or transmission
spectrum.  Its series equal the oracle's (the same reduction order) bit for
bit in FP64.  The probe spectra of a session accumulate on the GPU as the
steps run: in FP64 they are rfsyn's running sums (the oracle sums as rfsyn's
probe_dft_record does; they agree to 1e-12, the device's sincos against
libm's); in FP32 (Kahan sums, FP64 phase recurrence) they stay within 1e-6
of the same transform of the stored FP32 series.  Physics pin: a plane wave
on a dielectric half-space (eps_r 4) reflects |R(f)| = 1/3 (within 0.02)
across the band, from the reflection plane's running spectrum against the
incident plane's."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from rfsyn_b200 import scenes
from tests.cases import DT1, workload_to_scene

pytestmark = pytest.mark.gpu


def _c3(precision):
    return scenes.c3(seed=7, precision=precision, nx=12, ny=10, nz=96, n_steps=600, npml=6, grid_probes=2)


def test_plane_series_and_spectra_equal_the_oracle_in_fp64():
    w = _c3(rb.FP64)
    want = oracle.run_oracle(workload_to_scene(w, slab_source="product"))
    st = scenes.scene_setup(w)
    got = rb.run(scenes.run_config(w), st.ptr, None)
    assert got["td"].shape[0] == len(w.probes) + len(w.planes) == want["td"].shape[0]
    assert np.array_equal(got["td"], want["td"])
    scale = np.abs(want["dft"]).max(axis=1, keepdims=True)
    assert float((np.abs(got["dft"] - want["dft"]) / scale).max()) <= 1e-12
    assert np.abs(want["td"][-4:]).max() > 0  # the planes see the wave


def _dft(series, freqs, dt, t_off=1.0):
    n = np.arange(series.shape[1])
    ph = np.exp(-1j * 2 * np.pi * np.outer(freqs, (n + t_off) * dt))
    return (series @ ph.T) * dt


def test_fp32_running_dft_matches_its_series():
    w = _c3(rb.FP32)
    st = scenes.scene_setup(w)
    sim = rb.Sim(scenes.run_config(w), st.ptr, None)
    try:
        sim.advance(w.n_steps)
        got = sim.dft()
        td = sim.probes()
    finally:
        sim.close()
    want = _dft(td, np.asarray(w.freqs), w.dt)
    err = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
    assert err.max() <= 1e-6, err.max()


def _half_space(precision, eps, plane_k, nz=400, kz0=60, kint=200):
    freqs = list(np.linspace(2e9, 12e9, 41))
    rc = rb.RunConfig(4, 4, nz, 1e-3, 1000, 10, periodic=3, precision=precision,
                      plane_wave=dict(theta=0.0, phi=0.0, psi=0.0, amplitude=1.0, i0=0, i1=3, j0=0, j1=3,
                                      k0=kz0, k1=nz - 30, waveform=rb.WAVE_GAUSSIAN_DERIV, p0=80 * DT1,
                                      p1=20 * DT1, p2=0.0),
                      freqs=freqs, planes=[dict(axis=2, index=plane_k, component=rb.FIELD_EX)])
    st = rb.SceneSetup(boxes=[(0, 4, 0, 4, kint, nz - 10, eps, 0.0)]) if eps != 1.0 else None
    return rb.run(rc, st.ptr if st else None, None)["dft"][0]


@pytest.mark.parametrize("precision", [rb.FP64, rb.FP32], ids=["fp64", "fp32"])
def test_fresnel_reflection_spectrum_from_plane_probes(precision):
    refl = _half_space(precision, 4.0, 50)      # scattered region below the boundary
    inc = _half_space(precision, 1.0, 200)      # incident wave where the interface will be
    band = np.abs(inc) > 0.2 * np.abs(inc).max()
    r = np.abs(refl[band]) / np.abs(inc[band])
    assert band.sum() >= 10
    assert np.all(np.abs(r - 1.0 / 3.0) < 0.02), r
