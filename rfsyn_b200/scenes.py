"""Seeded synthetic workloads of the FDTD stage.

All randomness comes from PCG32 exactly as rfsyn seeds its streams
(engine/core/rng.c:3-23: state 0, inc = stream<<1 | 1, one step, add the
seed, one step), so every scene is reproducible from (seed, stream).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import C0, FIELD_EX, FIELD_EY, FIELD_EZ, FP32, FP64, FUSED, WAVE_MOD_GAUSSIAN

M64 = (1 << 64) - 1


class Pcg32:
    """PCG32 (XSH-RR), rfsyn's rng_seed / rng_next_u32 / rng_uniform."""

    def __init__(self, seed: int, stream: int = 0):
        self.state = 0
        self.inc = ((stream << 1) | 1) & M64
        self.next_u32()
        self.state = (self.state + seed) & M64
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * 6364136223846793005 + self.inc) & M64
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((-rot) & 31))) & 0xFFFFFFFF

    def uniform(self) -> float:
        """[0, 1) with 24 bits, as rng_uniform."""
        return float(self.next_u32() >> 8) / float(1 << 24)

    def randint(self, lo: int, hi: int) -> int:
        """Integer in [lo, hi)."""
        return lo + self.next_u32() % (hi - lo)

    def range(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.uniform()

    def log_range(self, lo: float, hi: float) -> float:
        return math.exp(math.log(lo) + (math.log(hi) - math.log(lo)) * self.uniform())


def dt_of(dx: float, courant: float = 0.99) -> float:
    return courant * (dx / (C0 * math.sqrt(3.0)))


@dataclass
class Workload:
    """A full run description: grid, CPML, sources, probes, DFT bins."""

    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    n_steps: int
    npml: int
    kappa_max: float = 7.0
    m: float = 3.0
    ma: float = 1.0
    alpha_max: float = 0.05
    r0: float = 1e-6
    courant: float = 0.99
    periodic: int = 0
    precision: int = FP64
    schedule: int = FUSED
    sources: list = field(default_factory=list)   # dicts: i j k component mode amplitude waveform p0 p1 p2
    probes: list = field(default_factory=list)    # dicts: i j k component
    planes: list = field(default_factory=list)    # plane probes, dicts: axis index component
    freqs: list = field(default_factory=list)
    # scene pieces applied by a setup callback: boxes, component overrides
    boxes: list = field(default_factory=list)     # (i0,i1,j0,j1,k0,k1,eps,sigma)
    comps: list = field(default_factory=list)     # (comp,i,j,k,eps,sigma)
    # spheres (cx, cy, cz, radius, eps_r, sigma, model) in cell units; model is
    # None or (eps_inf, sigma, poles) with poles as in rfsyn_b200.dispersive
    spheres: list = field(default_factory=list)
    smoothing: int = 1
    # staircased anisotropic slabs (point[3], normal[3], thickness, eps_r 3x3),
    # dispersive boxes (i0,i1,j0,j1,k0,k1, model as for spheres), a plane wave
    slabs: list = field(default_factory=list)
    disp_boxes: list = field(default_factory=list)
    plane_wave: dict | None = None
    # slabs: 0 staircased, 1 faces smoothed (fdtd_b200_materials_set_tensor3_slab_smoothed)
    slab_smoothing: int = 0

    @property
    def dt(self) -> float:
        return dt_of(self.dx, self.courant)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def c1(seed: int = 1, precision: int = FP64) -> Workload:
    """Plain FDTD, 64^3 vacuum, dx 1 mm, 10-cell CPML (m 3, kappa_max 5,
    alpha 0.05 -> 0 with ma 1, r0 1e-6), soft Ez point source at the centre
    with a Gaussian-modulated sinusoid f0 10 GHz whose envelope exp(-u^2),
    u = (t-t0)/tau, has tau = 2/(pi 8 GHz) (1/e spectral full width 8 GHz)
    and t0 = 4 tau; 1000 steps; 4 Ez probes at PCG32(seed, 0) interior
    positions in [npml+2, 64-npml-2); 64 DFT bins linear over 2..18 GHz."""
    n, npml = 64, 10
    tau = 2.0 / (math.pi * 8e9)
    rng = Pcg32(seed, 0)
    lo, hi = npml + 2, n - npml - 2
    probes = [dict(i=rng.randint(lo, hi), j=rng.randint(lo, hi), k=rng.randint(lo, hi), component=FIELD_EZ)
              for _ in range(4)]
    return Workload(
        name="c1_64cube_fp64_vacuum", nx=n, ny=n, nz=n, dx=1e-3, n_steps=1000, npml=npml, kappa_max=5.0,
        precision=precision,
        sources=[dict(i=32, j=32, k=32, component=FIELD_EZ, mode=0, amplitude=1.0, waveform=WAVE_MOD_GAUSSIAN,
                      p0=10e9, p1=4.0 * tau, p2=tau)],
        probes=probes, freqs=list(np.linspace(2e9, 18e9, 64)))


def c2(seed: int = 2, precision: int = FP32) -> Workload:
    """FP32 FDTD, 256^3, dx 0.5 mm, 12-cell CPML (rfsyn's default grading),
    24 PCG32(seed, 0) dielectric spheres (radius U[4,30] cells, eps_r
    U[1.5,12], sigma log-U[1e-4,1e-1] S/m) with subpixel-smoothed diagonal
    permittivity at their surfaces, then 3 single-pole Debye spheres (radius
    U[4,30], eps_inf U[2,4], delta_eps U[5,60], tau log-U[1e-11,1e-9] s),
    centres uniform where the sphere clears the CPML; 4000 steps; soft Ez
    source at the centre, Gaussian-modulated sinusoid f0 20 GHz, envelope
    tau = 2/(pi 16 GHz), t0 = 4 tau; 16 Ez probes at interior PCG32
    positions; 256 DFT bins linear over 4..36 GHz."""
    n, npml = 256, 12
    rng = Pcg32(seed, 0)
    spheres = []

    def centre(r):
        lo, hi = npml + r + 2, n - npml - r - 2
        return [rng.range(lo, hi) for _ in range(3)]

    for _ in range(24):
        r = rng.range(4.0, 30.0)
        c = centre(r)
        spheres.append((c[0], c[1], c[2], r, rng.range(1.5, 12.0), rng.log_range(1e-4, 1e-1), None))
    for _ in range(3):
        r = rng.range(4.0, 30.0)
        c = centre(r)
        model = (rng.range(2.0, 4.0), 0.0, [("debye", rng.range(5.0, 60.0), rng.log_range(1e-11, 1e-9))])
        spheres.append((c[0], c[1], c[2], r, 1.0, 0.0, model))
    lo, hi = npml + 2, n - npml - 2
    probes = [dict(i=rng.randint(lo, hi), j=rng.randint(lo, hi), k=rng.randint(lo, hi), component=FIELD_EZ)
              for _ in range(16)]
    tau = 2.0 / (math.pi * 16e9)
    return Workload(
        name="c2_256cube_fp32_24spheres_3debye", nx=n, ny=n, nz=n, dx=0.5e-3, n_steps=4000, npml=npml,
        precision=precision,
        sources=[dict(i=n // 2, j=n // 2, k=n // 2, component=FIELD_EZ, mode=0, amplitude=1.0,
                      waveform=WAVE_MOD_GAUSSIAN, p0=20e9, p1=4.0 * tau, p2=tau)],
        probes=probes, freqs=list(np.linspace(4e9, 36e9, 256)), spheres=spheres)


def c4(seed: int = 4, n_scenes: int = 512, precision: int = FP32, n_steps: int = 1500,
       lo: int = 32, hi: int = 96, npml: int = 8) -> list[Workload]:
    """Batched FDTD: n_scenes independent scenes, per-axis sizes uniform in
    [lo, hi] cells, dx 1 mm, 8-cell CPML (rfsyn's default grading); 0-6
    scatterers per scene, each a sphere (radius U[3,12] cells) or a box (sides
    U[4,16] cells) with eps_r U[1,10] and sigma log-U[1e-4,1] S/m, clear of
    the CPML (radii and sides capped to fit the smallest axis); one soft Ez dipole (Gaussian-modulated sinusoid f0 10 GHz,
    tau = 2/(pi 8 GHz), t0 = 4 tau) and 4 Ez probes at interior positions;
    n_steps steps; 128 DFT bins linear over 2..18 GHz.  Scene s draws from
    PCG32(seed, stream s).  Needs lo >= 2 npml + 12."""
    if lo < 2 * npml + 12:
        raise ValueError("c4: the smallest axis must leave room for scatterers between the CPML slabs")
    tau = 2.0 / (math.pi * 8e9)
    freqs = list(np.linspace(2e9, 18e9, 128))
    out = []
    for sc in range(n_scenes):
        rng = Pcg32(seed, sc)
        nx, ny, nz = (rng.randint(lo, hi + 1) for _ in range(3))
        dims = (nx, ny, nz)
        boxes, spheres = draw_scatterers(rng, dims, npml)
        m = npml + 3

        def pick():
            return [rng.randint(m, n - m) for n in dims]

        s = pick()
        probes = [dict(zip("ijk", pick()), component=FIELD_EZ) for _ in range(4)]
        out.append(Workload(
            name=f"c4_scene{sc}", nx=nx, ny=ny, nz=nz, dx=1e-3, n_steps=n_steps, npml=npml, precision=precision,
            sources=[dict(i=s[0], j=s[1], k=s[2], component=FIELD_EZ, mode=0, amplitude=1.0,
                          waveform=WAVE_MOD_GAUSSIAN, p0=10e9, p1=4.0 * tau, p2=tau)],
            probes=probes, freqs=freqs, boxes=boxes, spheres=spheres))
    return out


def draw_scatterers(rng: Pcg32, dims, npml: int) -> tuple[list, list]:
    """0-6 scatterers clear of the CPML, each a sphere (radius U[3,12] cells)
    or a box (sides U[4,16] cells) with eps_r U[1,10] and sigma log-U[1e-4,1]
    S/m (radii and sides capped to fit the smallest axis), drawn from rng.
    Returns (boxes, spheres) in the Workload's forms.  Needs
    min(dims) >= 2 npml + 12."""
    boxes, spheres = [], []
    room = min(dims) - 2 * (npml + 2)   # cells between the CPML margins
    for _ in range(rng.randint(0, 7)):
        eps, sig = rng.range(1.0, 10.0), rng.log_range(1e-4, 1.0)
        if rng.next_u32() & 1:
            r = rng.range(3.0, min(12.0, room / 2 - 1))
            c = [rng.range(npml + r + 2, n - npml - r - 2) for n in dims]
            spheres.append((c[0], c[1], c[2], r, eps, sig, None))
        else:
            b = []
            for n in dims:
                side = rng.randint(4, min(17, room))
                a0 = rng.randint(npml + 2, n - npml - 2 - side + 1)
                b += [a0, a0 + side]
            boxes.append((*b, eps, sig))
    return boxes, spheres


def scene_setup(w: Workload):
    """The workload's boxes, spheres, dispersive boxes and anisotropic slabs
    as a setup callback (None when it has none)."""
    if not (w.boxes or w.spheres or w.slabs or w.disp_boxes):
        return None
    from . import SceneSetup, dispersive

    rows = [(cx, cy, cz, r, eps, sig, None if model is None else dispersive(*model))
            for (cx, cy, cz, r, eps, sig, model) in w.spheres]
    return SceneSetup(w.boxes, rows, w.smoothing, slabs=w.slabs,
                      disp_boxes=[(*b[:6], dispersive(*b[6])) for b in w.disp_boxes], slab_smoothing=w.slab_smoothing)


def _gauss(rng: Pcg32) -> float:
    """Standard normal from two PCG32 uniforms (Box-Muller)."""
    u1 = max(rng.uniform(), 1e-12)
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * rng.uniform())


def c3(seed: int = 3, precision: int = FP32, nx: int = 128, ny: int = 128, nz: int = 512, n_steps: int = 6000,
       npml: int = 16, dx: float = 0.5e-3, grid_probes: int = 8, slab_smoothing: int = 1) -> Workload:
    """Periodic unit cell nx x ny x nz (periodic x / y, npml-cell CPML in z),
    dx 0.5 mm.  A plane wave at normal incidence (a non-normal wave is not
    periodic in x / y) with a PCG32(seed) polarisation angle, through a TF/SF
    boundary 4 cells inside the CPML; a Gaussian-modulated sinusoid f0 12 GHz,
    tau = 2/(pi 16 GHz), t0 = 4 tau.  One tilted slab (seeded normal within
    45 deg of z, thickness U[20,60] cells, centred at 0.55 nz) of a full 3x3
    eps_r: eigenvalues U[2,10] rotated by the QR factor of a seeded Gaussian
    matrix, its faces subpixel-smoothed (slab_smoothing 1; 0 staircases
    them).  A 12-cell 2-pole Lorentz layer at 0.3 nz (f_p U[5,20] GHz,
    gamma 2 pi U[0.1,1] GHz, delta_eps U[0.5,3]).  Reflection plane (in the
    scattered region below the boundary) and transmission plane (near the
    top): each a plane probe of Ex and one of Ey (the mean over the whole
    plane, the specular wave) and grid_probes^2 Ex point probes; 512 DFT bins
    over 2..24 GHz, accumulated as the steps run; n_steps steps.  Series:
    the 2 grid_probes^2 point probes, then the planes (reflection Ex, Ey,
    transmission Ex, Ey)."""
    rng = Pcg32(seed, 0)
    psi = rng.range(0.0, math.pi)
    th, ph = rng.range(0.0, math.pi / 4), rng.range(0.0, 2.0 * math.pi)
    normal = [math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)]
    thick = rng.range(20.0, 60.0)
    lam = [rng.range(2.0, 10.0) for _ in range(3)]
    G = np.array([[_gauss(rng) for _ in range(3)] for _ in range(3)])
    Q, _ = np.linalg.qr(G)
    eps = Q @ np.diag(lam) @ Q.T
    eps = 0.5 * (eps + eps.T)
    poles = [("lorentz", rng.range(0.5, 3.0), 2.0 * math.pi * rng.range(5e9, 20e9),
              2.0 * math.pi * rng.range(0.1e9, 1e9)) for _ in range(2)]
    zl = int(0.3 * nz)
    tau = 2.0 / (math.pi * 16e9)
    k0, k1 = npml + 4, nz - npml - 4
    pw = dict(theta=0.0, phi=0.0, psi=psi, amplitude=1.0, waveform=WAVE_MOD_GAUSSIAN, p0=12e9, p1=4.0 * tau,
              p2=tau, i0=0, i1=nx - 1, j0=0, j1=ny - 1, k0=k0, k1=k1)
    g = grid_probes
    pts = [(int((a + 0.5) * nx / g), int((b + 0.5) * ny / g)) for a in range(g) for b in range(g)]
    probes = [dict(i=i, j=j, k=npml + 2, component=FIELD_EX) for (i, j) in pts]
    probes += [dict(i=i, j=j, k=k1 - 8, component=FIELD_EX) for (i, j) in pts]
    planes = [dict(axis=2, index=k, component=c) for k in (npml + 2, k1 - 8) for c in (FIELD_EX, FIELD_EY)]
    return Workload(
        name=f"c3_{nx}x{ny}x{nz}_periodic_tfsf_aniso_lorentz", nx=nx, ny=ny, nz=nz, dx=dx, n_steps=n_steps,
        npml=npml, periodic=3, precision=precision, probes=probes, planes=planes,
        freqs=list(np.linspace(2e9, 24e9, 512)),
        slabs=[([0.5 * nx, 0.5 * ny, 0.55 * nz], normal, thick, eps.ravel().tolist())],
        disp_boxes=[(0, nx, 0, ny, zl, zl + 12, (1.0, 0.0, poles))], plane_wave=pw, slab_smoothing=slab_smoothing)


def scaled(w: Workload, n: int, n_steps: int) -> Workload:
    """The same scene recipe on an n^3 grid (spheres, probes and source scaled
    with the grid) for parity checks at oracle-friendly sizes."""
    f = n / w.nx
    npml = max(2, int(round(w.npml * f)))
    sp = []
    for (cx, cy, cz, r, eps, sig, model) in w.spheres:
        sp.append((cx * f, cy * f, cz * f, max(1.2, r * f), eps, sig, model))
    pr = [dict(i=min(n - 2, max(1, int(p["i"] * f))), j=min(n - 2, max(1, int(p["j"] * f))),
               k=min(n - 2, max(1, int(p["k"] * f))), component=p["component"]) for p in w.probes]
    src = [dict(s, i=n // 2, j=n // 2, k=n // 2) for s in w.sources]
    return Workload(name=w.name + f"_scaled{n}", nx=n, ny=n, nz=n, dx=w.dx, n_steps=n_steps, npml=npml,
                    kappa_max=w.kappa_max, precision=w.precision, schedule=w.schedule, sources=src, probes=pr,
                    freqs=list(w.freqs), spheres=sp, smoothing=w.smoothing)


def sphere_setup(w: Workload):
    """The workload's spheres as a setup callback (None when it has none)."""
    if not w.spheres:
        return None
    from . import SphereSetup, dispersive

    rows = []
    for (cx, cy, cz, r, eps, sig, model) in w.spheres:
        rows.append((cx, cy, cz, r, eps, sig, None if model is None else dispersive(*model)))
    return SphereSetup(rows, w.smoothing)


def run_config(w: Workload):
    """The workload as an fdtd_b200_config_t (RunConfig)."""
    from . import CpmlParams, RunConfig

    return RunConfig(w.nx, w.ny, w.nz, w.dx, w.n_steps, w.npml, courant=w.courant, periodic=w.periodic,
                     precision=w.precision, schedule=w.schedule,
                     cpml=CpmlParams(w.npml, w.m, w.ma, w.kappa_max, w.alpha_max, w.r0),
                     sources=w.sources, probes=w.probes, freqs=w.freqs, plane_wave=w.plane_wave, planes=w.planes)
