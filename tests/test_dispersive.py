"""Dispersive (ADE) samples and smoothed spheres: features with no rfsyn
counterpart.  The CPU oracle restates them (oracle/fdtd_oracle.c) and is
pinned by physics: the static limit (delta_eps -> 0 reproduces a plain
eps_inf medium), the reflection of a plane wave from Debye / Lorentz
half-spaces against Fresnel with eps(omega), the field energy of passive
dispersive media in a closed box (never growing, decaying), and the sphere
fill fractions' volume partition, their known answers (half, quarter and
three-eighths cubes, 0 / 1 beyond the half diagonal, the squared normal)
and their z-invariant limit against rfsyn's 2-D square share
(subpixel_te_rectangle_fraction).  The GPU paths are held bit-for-bit to
the oracle in FP64."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle import MODEL_ONLY, Scene, disp_entry
from tests.cases import run_device

DT = Scene(nx=1, ny=1, nz=1).dt
BASE = dict(nx=16, ny=14, nz=12, n_steps=80, npml=3, sources=[(8, 7, 6, 2, 0, 1.0, 0, 20 * DT, 5 * DT, 0)],
            probes=[(11, 7, 6, 2), (8, 9, 6, 0), (6, 5, 4, 1)], freqs=[20e9, 45e9])

DEBYE = ("debye", 20.0, 3e-11)
LORENTZ = ("lorentz", 3.0, 2 * math.pi * 12e9, 2 * math.pi * 0.5e9)

SCENES = {
    "debye_box": Scene(**BASE, disp=[disp_entry(c, i, j, k, 2.5, 0.0, [DEBYE])
                                     for c in range(3) for i in range(4, 12) for j in range(3, 11) for k in range(3, 9)]),
    "lorentz_debye_slab_lossy": Scene(**BASE, disp=[disp_entry(c, i, j, k, 2.0, 0.01, [LORENTZ, ("debye", 5.0, 1e-10)])
                                                    for c in range(3) for i in range(2, 15) for j in range(1, 13)
                                                    for k in range(6, 8)]),
    "spheres_smoothed": Scene(**BASE, disp=[disp_entry(0, MODEL_ONLY, 0, 0, 2.5, 0.0, [DEBYE]),
                                            disp_entry(0, MODEL_ONLY, 0, 0, 2.0, 0.01, [LORENTZ])],
                              spheres=[(8.3, 7.1, 6.2, 3.7, 6.0, 0.01, -1), (5.0, 5.0, 5.0, 2.2, 1.0, 0.0, 0),
                                       (10.5, 9.0, 7.0, 2.5, 1.0, 0.0, 1), (7.0, 4.0, 8.0, 2.9, 3.5, 0.0, -1)]),
    "spheres_staircase": Scene(**BASE, smoothing=0, spheres=[(8.3, 7.1, 6.2, 3.7, 6.0, 0.01, -1),
                                                             (7.6, 6.0, 5.5, 2.4, 11.0, 0.0, -1)]),
}


def test_oracle_debye_static_limit():
    # Debye with delta_eps -> 0 is a plain eps_inf medium
    a = oracle.run_oracle(Scene(**BASE, boxes=[(4, 12, 3, 11, 3, 9, 3.0, 0.0)]))
    b = oracle.run_oracle(Scene(**BASE, disp=[disp_entry(c, i, j, k, 3.0, 0.0, [("debye", 1e-9, 1e-11)])
                                              for c in range(3) for i in range(4, 12) for j in range(3, 11)
                                              for k in range(3, 9)]))
    assert np.abs(a["td"] - b["td"]).max() <= 1e-8 * np.abs(a["td"]).max()


def test_oracle_lorentz_static_limit():
    a = oracle.run_oracle(Scene(**BASE, boxes=[(4, 12, 3, 11, 3, 9, 2.0, 0.0)]))
    b = oracle.run_oracle(Scene(**BASE, disp=[disp_entry(c, i, j, k, 2.0, 0.0, [("lorentz", 1e-9, 2e11, 1e9)])
                                              for c in range(3) for i in range(4, 12) for j in range(3, 11)
                                              for k in range(3, 9)]))
    assert np.abs(a["td"] - b["td"]).max() <= 1e-8 * np.abs(a["td"]).max()


def test_oracle_debye_raises_low_frequency_delay():
    # a Debye medium is slower at low frequency (eps_s = eps_inf + delta_eps)
    # than its eps_inf limit: the pulse through it arrives later
    s_inf = Scene(**{**BASE, "n_steps": 140}, boxes=[(4, 13, 0, 15, 0, 13, 2.5, 0.0)])
    s_deb = Scene(**{**BASE, "n_steps": 140}, disp=[disp_entry(c, i, j, k, 2.5, 0.0, [("debye", 20.0, 1e-9)])
                                                  for c in range(3) for i in range(4, 13) for j in range(0, 15)
                                                  for k in range(0, 13)])
    a = oracle.run_oracle(s_inf)["td"][0]
    b = oracle.run_oracle(s_deb)["td"][0]
    assert np.argmax(np.abs(b)) >= np.argmax(np.abs(a))


EPS0 = 8.8541878128e-12
HALF_SPACES = {
    "debye": ([("debye", 4.0, 1 / (2 * math.pi * 3e9))], 2.0, 0.0),
    "lorentz": ([("lorentz", 2.0, 2 * math.pi * 12e9, 2 * math.pi * 1e9)], 2.0, 0.0),
    "debye_lorentz_lossy": ([("debye", 4.0, 1 / (2 * math.pi * 3e9)),
                             ("lorentz", 1.5, 2 * math.pi * 11e9, 2 * math.pi * 0.5e9)], 2.0, 0.005),
}


def half_space_scenes(poles, eps_inf, sigma, nz=600, kz0=60, kint=200, ks=50, n_steps=900):
    """Normal-incidence plane wave (TF/SF, periodic x / y) onto a dispersive
    half-space filling z >= kint (the interface sits between the E_x samples
    kint - 1 and kint, at z = kint - 1/2).  Scene a records the reflected
    E_x at z = ks in the scattered-field region; scene b (vacuum) records the
    incident E_x at the mirror point 2 (kint - 1/2) - ks, which has travelled
    exactly as far on the same grid.  The medium ends 10 cells inside the
    total-field box (the box boundary must lie in scalar media); the record
    ends before the wave reaches that far face."""
    pw = dict(theta=0.0, phi=0.0, psi=0.0, amplitude=1.0, i0=0, i1=3, j0=0, j1=3, k0=kz0, k1=nz - 30,
              waveform=0, p0=80 * DT, p1=20 * DT, p2=0.0)
    disp = [disp_entry(c, i, j, k, eps_inf, sigma, poles)
            for c in range(3) for i in range(4) for j in range(4) for k in range(kint, nz - 40)]
    base = dict(nx=4, ny=4, nz=nz, n_steps=n_steps, periodic=3, npml=10, plane_wave=pw)
    return (Scene(**base, disp=disp, probes=[(1, 1, ks, 0)]),
            Scene(**base, probes=[(1, 1, 2 * kint - 1 - ks, 0)]))


def fresnel(poles, eps_inf, sigma, f):
    """r = (1 - n) / (1 + n), n = sqrt(eps(omega)) for the e^{j omega t}
    convention: Debye delta_eps / (1 + j omega tau); Lorentz
    delta_eps wp^2 / (wp^2 - omega^2 + 2 j gamma omega) (the ADE
    J'' + 2 gamma J' + wp^2 J = eps0 delta_eps wp^2 E'); conductivity
    sigma / (j omega eps0)."""
    w = 2 * math.pi * f
    eps = np.full(f.shape, eps_inf, complex)
    for p in poles:
        eps += p[1] / (1 + 1j * w * p[2]) if p[0] == "debye" else p[1] * p[2] ** 2 / (p[2] ** 2 - w ** 2 + 2j * p[3] * w)
    eps += sigma / (1j * w * EPS0)
    n = np.sqrt(eps)
    return (1 - n) / (1 + n)


@pytest.mark.parametrize("name", sorted(HALF_SPACES))
def test_oracle_dispersive_half_space_matches_fresnel(name):
    poles, eps_inf, sigma = HALF_SPACES[name]
    a, b = half_space_scenes(poles, eps_inf, sigma)
    refl = oracle.run_oracle(a)["td"][0]
    inc = oracle.run_oracle(b)["td"][0]
    f = np.fft.rfftfreq(8192, a.dt)
    got = np.fft.rfft(refl, 8192) / np.fft.rfft(inc, 8192)
    lo, band = (f >= 1e9) & (f <= 3e9), (f >= 1e9) & (f <= 8e9)
    want = fresnel(poles, eps_inf, sigma, f[band])
    err = np.abs(got[band] - want)
    # complex r within 2e-3 where the grid has > 40 cells per wavelength in
    # the medium, 1e-2 up to 8 GHz (Yee dispersion grows as (k dx)^2)
    assert err[lo[band]].max() < 2e-3, err[lo[band]].max()
    assert err.max() < 1e-2, err.max()


@pytest.mark.gpu
def test_device_fp64_dispersive_half_space_equals_oracle():
    poles, eps_inf, sigma = HALF_SPACES["debye_lorentz_lossy"]
    a, _ = half_space_scenes(poles, eps_inf, sigma)
    a.probes = [(1, 1, 50, 0), (2, 2, 260, 0), (0, 3, 400, 1)]
    want = oracle.run_oracle(a)
    got = run_device(a, rb.FP64, rb.FUSED)
    assert np.array_equal(got["td"], want["td"])


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [rb.SPLIT, rb.FUSED])
@pytest.mark.parametrize("name", sorted(SCENES))
def test_device_fp64_matches_oracle_bit_exact(name, schedule):
    s = SCENES[name]
    want = oracle.run_oracle(s)
    got = run_device(s, rb.FP64, schedule)
    assert np.array_equal(got["td"], want["td"]), np.abs(got["td"] - want["td"]).max()
    assert np.linalg.norm(got["dft"] - want["dft"]) <= 1e-12 * np.linalg.norm(want["dft"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SCENES))
def test_device_fp32_close_to_oracle(name):
    s = SCENES[name]
    want = oracle.run_oracle(s)
    got = run_device(s, rb.FP32, rb.FUSED)
    for p in range(want["td"].shape[0]):
        scale = np.abs(want["td"][p]).max()
        assert np.abs(got["td"][p] - want["td"][p]).max() <= 1e-3 * scale


@pytest.mark.gpu
def test_sphere_fractions_partition_volume():
    # the fractions of all E_z samples of a sphere sum to its volume
    # (each sample owns one unit cube); 8^3 supersampling error is small
    import ctypes as C

    lib = rb.load()
    f = lib.rfb_sphere_fractions
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_double), C.c_double] + [C.c_int] * 6 + [C.POINTER(C.c_double)] * 2
    r = 7.3
    n = 24
    cen = (C.c_double * 3)(12.2, 11.9, 12.4)
    fr = np.zeros(3 * n ** 3)
    n2 = np.zeros(3 * n ** 3)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    assert f(cen, r, 0, 0, 0, n, n, n, dp(fr), dp(n2)) == 0
    vol = 4.0 / 3.0 * math.pi * r ** 3
    for c in range(3):
        assert abs(fr[c::3].sum() - vol) / vol < 2e-3
    assert fr.min() >= 0.0 and fr.max() <= 1.0


# ---- known answers of the fill fractions and a passivity pin ------------------------
# A sphere of radius 1e4 is a plane at the scale of one cell (its surface
# leaves the tangent plane by at most (sqrt(3)/2)^2 / 2e4 < 4e-5 cells over a
# cube), so with the centre placed at p + (d - R) n the sphere holds the
# points x near the sample p with n . (x - p) <= d.
_R = 1.0e4


def _fractions():
    import ctypes as C

    lib = rb.load()
    f = lib.rfb_sphere_fractions
    f.restype = C.c_int
    f.argtypes = [C.POINTER(C.c_double), C.c_double] + [C.c_int] * 6 + [C.POINTER(C.c_double)] * 2

    def plane(cell, comp, n, d):
        p = np.array(cell, dtype=float)
        p[comp] += 0.5
        cen = (C.c_double * 3)(*(p + (d - _R) * np.asarray(n, dtype=float)))
        fr, n2 = np.zeros(3), np.zeros(3)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        assert f(cen, _R, cell[0], cell[1], cell[2], 1, 1, 1, dp(fr), dp(n2)) == 0
        return fr[comp], n2[comp]

    return plane


_LAT = (np.arange(8) + 0.5) / 8 - 0.5  # lattice offsets of the 8^3 points


@pytest.mark.gpu
def test_sphere_fraction_known_answers():
    """Axis-aligned surfaces through and near the sample: half, quarter and
    three-eighths cubes exactly (lattice layers at odd sixteenths), 0 and 1
    beyond the half diagonal, and the squared normal of the sample's
    component exactly 1 or 0."""
    plane = _fractions()
    want = {0.0: 0.5, 0.25: 0.75, -0.25: 0.25, 0.375: 0.875, -0.375: 0.125, 0.9: 1.0, -0.9: 0.0}
    for comp in range(3):
        for axis in range(3):
            for sign in (1.0, -1.0):
                n = np.zeros(3)
                n[axis] = sign
                for d, fw in want.items():
                    fr, n2 = plane((7, 6, 5), comp, n, d)
                    assert fr == fw, (comp, axis, sign, d, fr)
                    assert n2 == (1.0 if axis == comp else 0.0)


@pytest.mark.gpu
def test_sphere_fraction_two_d_limit_against_subpixel_te():
    """A surface invariant along z: the cube's share is the 8 x 8 lattice
    count of the square cut by the line, exactly, and within the lattice's
    resolution of rfsyn's exact square share (subpixel_te_rectangle_fraction
    of a rectangle whose edge is that line)."""
    import ctypes as C

    from tests.test_subpixel import Rect, _bind

    plane = _fractions()
    lib = _bind(rb.load())
    rng = np.random.default_rng(21)
    diffs = []
    checked = 0
    while checked < 300:
        th, d = rng.uniform(-np.pi, np.pi), rng.uniform(-0.7, 0.7)
        n = np.array([np.cos(th), np.sin(th), 0.0])
        s = n[0] * _LAT[:, None] + n[1] * _LAT[None, :] - d
        if np.abs(s).min() < 1e-3:  # a lattice point on the line: the curvature decides it
            continue
        fr, n2 = plane((9, 9, 4), 2, n, d)
        assert fr == np.count_nonzero(s <= 0) / 64.0, (th, d, fr)
        assert n2 <= 1e-20  # Ez sample, normal in the (x, y) plane
        p2 = np.array([9.0, 9.0])
        cen = p2 + (d - 0.5 * _R) * n[:2]
        area = C.c_double()
        assert lib.subpixel_te_rectangle_fraction(C.byref(Rect(cen[0], cen[1], _R, _R, th)), p2[0], p2[1], 1.0, 1.0,
                                                  C.byref(area)) == 0
        diffs.append(abs(fr - area.value))
        checked += 1
    # an 8 x 8 lattice of a unit square cut by a straight line: at most one
    # point per lattice column or row misjudged, |error| <= 8 / 64
    assert max(diffs) <= 0.125 and np.mean(diffs) < 0.03, (max(diffs), np.mean(diffs))


@pytest.mark.gpu
def test_passive_dispersive_media_do_not_gain_energy():
    """A PEC box holding lossy Debye and damped Lorentz media (passive:
    delta_eps > 0, tau > 0, gamma > 0, sigma >= 0), excited by a short pulse
    and then left alone: the field energy never grows window over window
    (rfsyn's windowed-peak test, validate_long_term_stability.c:226-253,
    with a 5 % margin for beating) and decays as the media absorb it."""
    lorentz = ("lorentz", 3.0, 2 * math.pi * 12e9, 2 * math.pi * 2e9)
    debye = ("debye", 5.0, 3e-11)
    n_steps = 3000
    s = Scene(nx=20, ny=20, nz=20, n_steps=n_steps, npml=0,
              sources=[(10, 10, 10, 2, 0, 1.0, 0, 20 * DT, 5 * DT, 0)], probes=[(12, 10, 10, 2)],
              disp=[disp_entry(c, i, j, k, 2.0, 0.005, [lorentz, debye] if (i + j) % 2 else [debye])
                    for c in range(3) for i in range(4, 16) for j in range(4, 16) for k in range(4, 16)])
    for precision in (rb.FP64, rb.FP32):
        from tests.cases import scene_run_config

        import ctypes as C

        rc = scene_run_config(s, precision, rb.FUSED)
        cs = s.to_c()
        sim = rb.Sim(rc, oracle.device_setup(), C.cast(C.pointer(cs), C.c_void_p))
        energy = []
        try:
            for _ in range(n_steps // 10):
                sim.advance(10)
                e = sim.energy()
                energy.append(e["electric_j"] + e["magnetic_j"])
        finally:
            sim.close()
        energy = np.array(energy)
        assert np.all(np.isfinite(energy)) and energy.max() > 0
        tail = energy[10:]  # the pulse ends by step 50
        peaks = tail[: len(tail) // 29 * 29].reshape(-1, 29).max(axis=1)  # windows of 290 steps
        assert np.all(peaks[1:] <= 1.05 * peaks[:-1]), (precision, peaks)
        assert peaks[-1] <= 0.5 * peaks[0], (precision, peaks)
