"""Oblique plane-wave incidence on a cell periodic across the wave's
transverse axes: the FP64 oracle of the fixed-transverse-wavenumber
formulation (Bloch-periodic complex fields, a 1-D incident line whose
transverse derivatives are the grid's own) pinned by physics.  CPU only:
the formulation's device path is not built."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import floquet_oracle as fo


def _cell(nx, ny, nz, f_cut, phi, d=0.5e-3):
    kt = 2.0 * math.pi * f_cut / fo.C0
    return fo.ObliqueCell(nx=nx, ny=ny, nz=nz, d=d, kx=kt * math.cos(phi), ky=kt * math.sin(phi))


@pytest.mark.parametrize("pol", ["te", "tm"])
@pytest.mark.parametrize("f_cut,phi", [(0.0, 0.0), (3e9, 0.0), (6e9, 0.4), (9e9, 2.2)])
def test_bloch_tfsf_leaves_nothing_in_vacuum(pol, f_cut, phi):
    """In vacuum the scattered region stays empty to rounding at every angle
    and azimuth (the line's amplitudes times the transverse phases are the
    cell's field exactly), with the Bloch wraps of both transverse axes in
    use (3 x 2 cells across)."""
    cell = _cell(3, 2, 240, f_cut, phi)
    r = fo.run(cell, np.ones(cell.nz + 1), pol, 700, k_src=30, k_rec=70, k_tf=90, f0=14e9,
               tau=2.0 / (math.pi * 8e9))
    assert r.leak < 1e-12, r.leak
    assert np.abs(r.inc_t).max() > 0.1


@pytest.mark.parametrize("pol", ["te", "tm"])
def test_oblique_reflection_matches_fresnel(pol):
    """An eps 4 half-space under a fixed transverse wavenumber (cut-off 6
    GHz, azimuth 0.4 rad): each frequency meets it at its own angle,
    sin(theta) = 6 GHz / f (33-21 deg over 11-17 GHz), and |R(f)| of the
    tangential E follows Fresnel's TE or TM coefficient within 0.02.  The run
    ends before the incident line's wall echo reaches the record plane."""
    cell = _cell(2, 1, 2000, 6e9, 0.4)
    er = np.ones(cell.nz + 1)
    er[900:] = 4.0
    r = fo.run(cell, er, pol, 4400, k_src=300, k_rec=800, k_tf=820, f0=14e9, tau=2.0 / (math.pi * 8e9))
    kt = math.hypot(cell.kx, cell.ky)
    # tangential E direction: z x kt for TE, along kt for TM
    v = np.array([-cell.ky, cell.kx]) / kt if pol == "te" else np.array([cell.kx, cell.ky]) / kt
    freqs = np.linspace(11e9, 17e9, 7)
    R = fo.spectrum(r.refl_t @ v, r.dt, freqs) / fo.spectrum(r.inc_t @ v, r.dt, freqs)
    sin_t = kt * fo.C0 / (2.0 * math.pi * freqs)
    F = fo.fresnel(pol, 4.0, sin_t)
    assert np.all(np.abs(np.abs(R) - np.abs(F)) < 0.02), (np.abs(R), np.abs(F))
    # the angles matter: at normal incidence both would read 1/3
    assert np.all(np.abs(np.abs(F) - 1.0 / 3.0) > 0.02)
