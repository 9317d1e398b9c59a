"""Test infrastructure (never on the product path): an FP64 numpy restatement
of oblique plane-wave incidence on a cell that is periodic across the
wave's transverse axes -- the formulation a GPU path for it follows.

Method: fixed transverse wavenumber (Bloch-periodic complex fields;
Aminian & Rahmat-Samii, "Spectral FDTD: a novel technique for the analysis
of oblique incident plane wave on periodic structures", IEEE Trans.
Antennas Propag. 54(6), 2006).  The fields are complex; every sample
carries the transverse dependence exp(-j (kx x + ky y)) across the period,
so the wrap of a periodic axis multiplies by a phase instead of copying:

    F(i + nx) = F(i) Px,   Px = exp(-j kx nx dx)   (likewise Py).

The Yee update itself is rfsyn's (real coefficients, applied to complex
fields).  At fixed (kx, ky) every frequency f sees the angle
sin(theta) = |kt| c / (2 pi f); below f = |kt| c / (2 pi) the wave is
evanescent.

Incident field: with the transverse dependence fixed, the grid's
difference operators act on it exactly: a difference across one cell of
exp(-j kx x), referred to the midpoint, is multiplication by -j Kx with
Kx = (2 / dx) sin(kx dx / 2).  The incident wave is therefore computed on a
1-D auxiliary line along z (same dz, dt and z staggering) whose transverse
derivatives are -j Kx and -j Ky; the 3-D grid carries exactly that line's
amplitudes times each component's transverse phase, so the total-field /
scattered-field corrections on the z planes leave nothing behind in
vacuum (to rounding) at any angle.  The line is driven by a current sheet:
an electric sheet along z x kt for TE (s) polarisation, a magnetic sheet
along z x kt for TM (p).

Grid: nx x ny x nz cells of size d, Yee staggering as rfsyn's (Ex at
(i+1/2, j, k), Hx at (i, j+1/2, k+1/2), ...), PEC walls at k = 0 and
k = nz; eps_r per z layer (laterally uniform media, so the Fresnel
coefficients are the closed-form check)."""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

C0 = 299792458.0
MU0 = 4e-7 * math.pi
EPS0 = 1.0 / (MU0 * C0 * C0)


@dataclass
class ObliqueCell:
    nx: int
    ny: int
    nz: int
    d: float
    kx: float
    ky: float
    courant: float = 0.5

    @property
    def dt(self) -> float:
        return self.courant * self.d / (C0 * math.sqrt(3.0))

    def kt_grid(self) -> tuple[float, float]:
        """Kx, Ky: the grid's transverse derivative factors."""
        return 2.0 / self.d * math.sin(self.kx * self.d / 2), 2.0 / self.d * math.sin(self.ky * self.d / 2)


def _phase(cell: ObliqueCell, comp: str) -> np.ndarray:
    """exp(-j (kx x + ky y)) at component comp's transverse positions,
    shape (nx, ny, 1)."""
    ox = 0.5 if comp in ("ex", "hy", "hz") else 0.0
    oy = 0.5 if comp in ("ey", "hx", "hz") else 0.0
    x = (np.arange(cell.nx) + ox) * cell.d
    y = (np.arange(cell.ny) + oy) * cell.d
    return np.exp(-1j * (cell.kx * x[:, None, None] + cell.ky * y[None, :, None]))


def _fwd(F: np.ndarray, axis: int, P: complex) -> np.ndarray:
    """F(i + 1) - F(i) along a Bloch-periodic axis."""
    Fp = np.roll(F, -1, axis=axis)
    idx = [slice(None)] * F.ndim
    idx[axis] = -1
    src = [slice(None)] * F.ndim
    src[axis] = 0
    Fp[tuple(idx)] = F[tuple(src)] * P
    return Fp - F


def _bwd(F: np.ndarray, axis: int, P: complex) -> np.ndarray:
    """F(i) - F(i - 1) along a Bloch-periodic axis."""
    Fm = np.roll(F, 1, axis=axis)
    idx = [slice(None)] * F.ndim
    idx[axis] = 0
    src = [slice(None)] * F.ndim
    src[axis] = -1
    Fm[tuple(idx)] = F[tuple(src)] * np.conj(P)
    return F - Fm


def _zf(F: np.ndarray) -> np.ndarray:
    """Forward z difference onto the half points k + 1/2 (k < nz): shape nz."""
    return F[..., 1:] - F[..., :-1]


def _zb(G: np.ndarray) -> np.ndarray:
    """Backward z difference of half-point values onto the integer points
    k = 1 .. nz - 1 (the walls stay zero): shape nz - 1."""
    return G[..., 1:] - G[..., :-1]


@dataclass
class Run:
    refl_t: np.ndarray       # (Ex, Ey) at (i, j) = (0, 0) of the record plane, scattered region, per step
    inc_t: np.ndarray        # the incident (Ex, Ey) at the same samples (auxiliary line)
    leak: float              # max |E| in the scattered region over the run / max |E_inc| there
    dt: float


def run(cell: ObliqueCell, eps_layers: np.ndarray, pol: str, n_steps: int, k_src: int, k_rec: int, k_tf: int,
        f0: float, tau: float) -> Run:
    """Runs the oblique cell: the 1-D auxiliary line (vacuum) driven at k_src
    by a Gaussian-modulated sinusoid sheet, and the 3-D Bloch cell fed
    through the TF/SF plane at k_tf (total field for E at k >= k_tf and H at
    k + 1/2 >= k_tf), recording the scattered tangential E at k_rec < k_tf.
    eps_layers[k] (nz + 1 values) is eps_r of the E samples at z index k
    (Ex, Ey at k; Ez at k + 1/2 takes layer k)."""
    assert pol in ("te", "tm") and 0 < k_src < k_rec < k_tf < cell.nz
    nx, ny, nz, d = cell.nx, cell.ny, cell.nz, cell.d
    dt = cell.dt
    Kx, Ky = cell.kt_grid()
    Px = np.exp(-1j * cell.kx * nx * d)
    Py = np.exp(-1j * cell.ky * ny * d)
    ce = dt / (EPS0 * d)
    ch = dt / (MU0 * d)
    er = np.asarray(eps_layers, dtype=np.float64)
    assert er.shape == (nz + 1,)
    kt = math.hypot(cell.kx, cell.ky)
    tx, ty = (-cell.ky / kt, cell.kx / kt) if kt > 0 else (0.0, 1.0)  # z x kt: TE's E, TM's H
    dx_, dy_ = -1j * Kx * d, -1j * Ky * d  # one cell's difference of the transverse dependence

    # auxiliary line amplitudes (vacuum): ex, ey at integer k, ez at k + 1/2;
    # hx, hy at k + 1/2, hz at integer k
    a_ex = np.zeros(nz + 1, complex); a_ey = np.zeros(nz + 1, complex); a_ez = np.zeros(nz, complex)
    a_hx = np.zeros(nz, complex); a_hy = np.zeros(nz, complex); a_hz = np.zeros(nz + 1, complex)
    shp = lambda n: (nx, ny, n)  # noqa: E731
    ex = np.zeros(shp(nz + 1), complex); ey = np.zeros(shp(nz + 1), complex); ez = np.zeros(shp(nz), complex)
    hx = np.zeros(shp(nz), complex); hy = np.zeros(shp(nz), complex); hz = np.zeros(shp(nz + 1), complex)
    ph = {c: _phase(cell, c)[..., 0] for c in ("ex", "ey", "hx", "hy")}
    q = k_tf - 1  # the H half-plane just below the boundary (scattered)

    def src(t):
        u = (t - 4.0 * tau) / tau
        return math.exp(-u * u) * math.sin(2.0 * math.pi * f0 * (t - 4.0 * tau))

    refl = np.zeros((n_steps, 2), complex)
    inc = np.zeros((n_steps, 2), complex)
    leak, inc_max = 0.0, 0.0
    for n in range(n_steps):
        # ---- H to n + 1/2: line, then cell (TF/SF: the scattered H at q
        # read the total E at k_tf) ----
        e_inc_x, e_inc_y = a_ex[k_tf], a_ey[k_tf]
        a_hx -= ch * (dy_ * a_ez - _zf(a_ey))
        a_hy -= ch * (_zf(a_ex) - dx_ * a_ez)
        a_hz -= ch * (dx_ * a_ey - dy_ * a_ex)
        if pol == "tm":  # magnetic current sheet along z x kt at k_src + 1/2
            s = src(n * dt)
            a_hx[k_src] += s * tx
            a_hy[k_src] += s * ty
        hx -= ch * (_fwd(ez, 1, Py) - _zf(ey))
        hy -= ch * (_zf(ex) - _fwd(ez, 0, Px))
        hz -= ch * (_fwd(ey, 0, Px) - _fwd(ex, 1, Py))
        hx[..., q] -= ch * e_inc_y * ph["ey"]
        hy[..., q] += ch * e_inc_x * ph["ex"]
        # ---- E to n + 1 (TF/SF: the total E at k_tf read the scattered H at q) ----
        a_ex[1:nz] += ce * (dy_ * a_hz[1:nz] - _zb(a_hy))
        a_ey[1:nz] += ce * (_zb(a_hx) - dx_ * a_hz[1:nz])
        a_ez += ce * (dx_ * a_hy - dy_ * a_hx)
        if pol == "te":  # electric current sheet along z x kt at k_src
            s = src((n + 0.5) * dt)
            a_ex[k_src] += s * tx
            a_ey[k_src] += s * ty
        ex[..., 1:nz] += ce / er[1:nz] * (_bwd(hz[..., 1:nz], 1, Py) - _zb(hy))
        ey[..., 1:nz] += ce / er[1:nz] * (_zb(hx) - _bwd(hz[..., 1:nz], 0, Px))
        ez += ce / er[:nz] * (_bwd(hy, 0, Px) - _bwd(hx, 1, Py))
        ex[..., k_tf] += ce / er[k_tf] * a_hy[q] * ph["hy"]
        ey[..., k_tf] -= ce / er[k_tf] * a_hx[q] * ph["hx"]
        refl[n] = ex[0, 0, k_rec], ey[0, 0, k_rec]
        inc[n] = a_ex[k_rec] * ph["ex"][0, 0], a_ey[k_rec] * ph["ey"][0, 0]
        inc_max = max(inc_max, float(np.abs(a_ex[:k_tf]).max()), float(np.abs(a_ey[:k_tf]).max()))
        leak = max(leak, float(np.abs(ex[..., :k_tf]).max()), float(np.abs(ey[..., :k_tf]).max()),
                   float(np.abs(ez[..., :q]).max()))
    return Run(refl_t=refl, inc_t=inc, leak=leak / inc_max if inc_max else 0.0, dt=dt)


def spectrum(series: np.ndarray, dt: float, freqs: np.ndarray) -> np.ndarray:
    """DFT of a sampled series at the given frequencies (weight dt)."""
    t = np.arange(series.shape[0]) * dt
    return (series[None, :] * np.exp(-2j * math.pi * freqs[:, None] * t[None, :])).sum(axis=1) * dt


def fresnel(pol: str, eps2: float, sin_t: np.ndarray) -> np.ndarray:
    """Reflection coefficient of the tangential E (TE) or tangential H (TM)
    from vacuum onto a half-space of eps2 (both non-magnetic)."""
    c1 = np.sqrt(1.0 - sin_t ** 2 + 0j)
    c2 = np.sqrt(eps2 - sin_t ** 2 + 0j)
    if pol == "te":
        return (c1 - c2) / (c1 + c2)
    return (eps2 * c1 - c2) / (eps2 * c1 + c2)
