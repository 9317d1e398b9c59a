"""Shared test scenes and converters between the oracle's scene description
and the product's run configuration."""
from __future__ import annotations

import ctypes as C
import dataclasses

import rfsyn_b200 as rb
from oracle import Scene
from rfsyn_b200 import scenes

DT1 = Scene(nx=1, ny=1, nz=1).dt  # dt at dx = 1 mm


def _gd(t0_steps, tau_steps, dt=DT1):
    return (0, t0_steps * dt, tau_steps * dt, 0.0)


CASES: dict[str, Scene] = {
    # CPML + boxes + per-component overrides + lossy media + two sources
    "cpml_materials": Scene(
        nx=20, ny=18, nz=16, n_steps=60, npml=4, kappa_max=5.0,
        boxes=[(5, 12, 4, 10, 3, 9, 4.0, 0.01), (8, 15, 9, 14, 6, 12, 2.5, 0.0)],
        comps=[(0, 6, 5, 4, 6.0, 0.02), (2, 7, 7, 7, 9.0, 0.0), (1, 10, 5, 8, 3.0, 0.1)],
        sources=[(10, 9, 8, 2, 0, 1.0, *_gd(30, 8)), (6, 6, 6, 0, 0, 0.5, 2, 10e9, 40 * DT1, 10 * DT1)],
        probes=[(14, 9, 8, 2), (5, 5, 5, 0), (12, 10, 9, 4)], freqs=[5e9, 10e9, 15e9]),
    # periodic y/z slab with rfsyn's 2x2 tensor edges (coupled neighbours)
    "periodic_tensor": Scene(
        nx=12, ny=10, nz=3, n_steps=80, periodic=6, npml=3,
        tensors=[(0, 5, 5, 1, 0.3, 0.05, 0.25), (1, 5, 5, 1, 0.25, 0.05, 0.3), (1, 6, 5, 1, 0.2, 0.04, 0.3),
                 (0, 5, 6, 1, 0.3, -0.02, 0.2), (1, 5, 6, 1, 0.3, 0.03, 0.2)],
        sources=[(4, 4, 1, 2, 0, 1.0, *_gd(20, 6))], probes=[(7, 5, 1, 2), (5, 5, 1, 0), (5, 5, 1, 1), (5, 5, 1, 5)]),
    # closed PEC box, no CPML; a hard source and a soft source on the padded
    # k = nz boundary plane (exercises the boundary sweep)
    "pec_boundary_sources": Scene(
        nx=12, ny=11, nz=10, n_steps=70,
        boxes=[(3, 8, 2, 6, 4, 9, 3.0, 0.0)],
        sources=[(6, 5, 10, 0, 0, 1.0, *_gd(15, 4)), (4, 4, 4, 2, 1, 1.0, 1, 40e9, 12 * DT1, 0.0)],
        probes=[(6, 6, 9, 0), (7, 5, 10, 5), (6, 5, 10, 0), (2, 2, 2, 2)]),
    # fully periodic, lossy box, many overrides on a vacuum background
    "periodic_all_overrides": Scene(
        nx=9, ny=8, nz=7, n_steps=50, periodic=7,
        boxes=[(2, 5, 2, 5, 2, 5, 1.0, 0.05)],
        comps=[(c, i, 3, 4, 2.0 + i, 0.0) for c in range(3) for i in range(1, 8)],
        sources=[(4, 4, 3, 1, 0, 1.0, *_gd(12, 3))], probes=[(0, 0, 0, 1), (8, 7, 6, 3), (4, 4, 3, 1)],
        freqs=[20e9, 40e9]),
    # periodic x only (the march wraps), CPML on y/z, source on an x-wrapped cell
    "periodic_x_cpml": Scene(
        nx=10, ny=14, nz=12, n_steps=60, periodic=1, npml=3,
        boxes=[(0, 10, 5, 9, 4, 8, 5.0, 0.001)],
        sources=[(10, 7, 6, 2, 0, 1.0, *_gd(18, 5))], probes=[(0, 7, 6, 2), (9, 3, 3, 3), (5, 8, 7, 1)]),
}


def simulate_unit_cfg() -> rb.FdtdSimConfig:
    """tests/simulate_unit.c:9-27 of rfsyn."""
    c = rb.FdtdSimConfig()
    c.nx = c.ny = c.nz = 50
    c.dx, c.courant_safety, c.n_steps, c.npml = 1e-3, 0.99, 200, 8
    c.src_i = c.src_j = c.src_k = 25
    c.src_component = rb.FIELD_EZ
    c.t0_over_dt, c.tau_over_dt = 40.0, 8.0
    c.probe_i, c.probe_j, c.probe_k = 31, 25, 25
    c.probe_component = rb.FIELD_EZ
    return c


def slab_rows(w: scenes.Workload) -> list:
    """The 3x3 rows the product's slab helper gives the workload's slabs, as
    the oracle's explicit samples (the staircased helper runs on the host;
    the smoothed one builds its rows on the GPU)."""
    return product_t3_rows(dataclasses.replace(w, boxes=[], spheres=[], disp_boxes=[]))


def product_t3_rows(w: scenes.Workload) -> list:
    """Every 3x3 sample the product's set-up of the workload creates (its
    materials built through the host API on a bare grid)."""
    lib = rb.load()
    lib.fdtd_grid_create.restype = C.c_void_p
    lib.fdtd_grid_create.argtypes = [C.c_size_t] * 3 + [C.c_double, C.c_double]
    lib.fdtd_grid_set_periodic.argtypes = [C.c_void_p, C.c_uint]
    lib.materials_create.restype = C.c_void_p
    lib.materials_create.argtypes = [C.c_void_p]
    lib.materials_destroy.argtypes = [C.c_void_p]
    lib.fdtd_grid_destroy.argtypes = [C.c_void_p]
    lib.fdtd_b200_materials_get_tensor3.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + [C.c_size_t] * 3 + \
        [C.POINTER(C.c_double)]
    g = lib.fdtd_grid_create(w.nx, w.ny, w.nz, w.dx, w.courant)
    lib.fdtd_grid_set_periodic(g, w.periodic)
    m = lib.materials_create(g)
    st = scenes.scene_setup(w)
    assert st is not None and st.fn(g, m, None) == 0
    rows = []
    row = (C.c_double * 3)()
    ext = [n + (0 if (w.periodic >> a) & 1 else 1) for a, n in enumerate((w.nx, w.ny, w.nz))]
    for i in range(ext[0]):
        for j in range(ext[1]):
            for k in range(ext[2]):
                for c in range(3):
                    if lib.fdtd_b200_materials_get_tensor3(m, g, c, i, j, k, row) == 0:
                        rows.append((c, i, j, k, tuple(row)))
    lib.materials_destroy(m)
    lib.fdtd_grid_destroy(g)
    return rows


def oracle_slab_rows(w: scenes.Workload) -> list:
    """The oracle's own rows of the workload's slabs (uniform vacuum
    background): the staircased rule, or the smoothed faces of
    oracle.subpixel_oracle.slab_rows."""
    from oracle.subpixel_oracle import slab_rows as smooth_rows

    rows = []
    for (point, normal, thick, eps) in w.slabs:
        if w.slab_smoothing:
            rows += smooth_rows(w.nx, w.ny, w.nz, w.periodic, point, normal, thick, eps)
        else:
            rows += slab_rows(dataclasses.replace(w, slabs=[(point, normal, thick, eps)]))
    return rows


def workload_to_scene(w: scenes.Workload, slab_source: str = "oracle") -> Scene:
    """The workload as the oracle's scene.  Slab samples: the oracle's own
    rows (slab_source "oracle"), or the rows the product's helper built
    ("product": a smoothed slab then needs the GPU)."""
    from oracle import MODEL_ONLY, disp_entry

    disp, spheres = [], []
    for (cx, cy, cz, r, eps, sig, model) in w.spheres:
        idx = -1
        if model is not None:
            idx = len(disp)
            disp.append(disp_entry(0, MODEL_ONLY, 0, 0, model[0], model[1], model[2]))
        spheres.append((cx, cy, cz, r, eps, sig, idx))
    sc = Scene(
        nx=w.nx, ny=w.ny, nz=w.nz, dx=w.dx, courant=w.courant, n_steps=w.n_steps, periodic=w.periodic,
        npml=w.npml, m=w.m, ma=w.ma, kappa_max=w.kappa_max, alpha_max=w.alpha_max, r0=w.r0,
        boxes=list(w.boxes), comps=list(w.comps), disp=disp, spheres=spheres, smoothing=w.smoothing,
        sources=[(s["i"], s["j"], s["k"], s["component"], s["mode"], s["amplitude"], s["waveform"], s["p0"],
                  s["p1"], s.get("p2", 0.0)) for s in w.sources],
        probes=[(p["i"], p["j"], p["k"], p["component"]) for p in w.probes], freqs=list(w.freqs),
        planes=[(p["axis"], p["index"], p["component"]) for p in w.planes],
        src_t_offset=0.0, dft_t_offset=1.0, plane_wave=w.plane_wave,
        tensor3=(slab_rows(w) if slab_source == "product" else oracle_slab_rows(w)) if w.slabs else [])
    for (i0, i1, j0, j1, k0, k1, model) in w.disp_boxes:
        for i in range(i0, i1):
            for j in range(j0, j1):
                for k in range(k0, k1):
                    for c in range(3):
                        sc.disp.append(disp_entry(c, i, j, k, model[0], model[1], model[2]))
    return sc


def c1_scene() -> Scene:
    return workload_to_scene(scenes.c1())


def scene_run_config(s: Scene, precision: int, schedule: int) -> rb.RunConfig:
    cp = rb.CpmlParams(s.npml, s.m, s.ma, s.kappa_max, s.alpha_max, s.r0)
    return rb.RunConfig(
        s.nx, s.ny, s.nz, s.dx, s.n_steps, s.npml, courant=s.courant, periodic=s.periodic, precision=precision,
        schedule=schedule, cpml=cp,
        sources=[dict(i=q[0], j=q[1], k=q[2], component=q[3], mode=q[4], amplitude=q[5], waveform=q[6], p0=q[7],
                      p1=q[8], p2=q[9]) for q in s.sources],
        probes=[dict(i=q[0], j=q[1], k=q[2], component=q[3]) for q in s.probes], freqs=s.freqs,
        source_time_offset=s.src_t_offset, dft_time_offset=s.dft_t_offset, plane_wave=s.plane_wave,
        planes=[dict(axis=a, index=i, component=c) for (a, i, c) in s.planes])


def run_device(s: Scene, precision: int, schedule: int) -> dict:
    """The product's device time loop on scene s (materials via scn_setup)."""
    import oracle

    rc = scene_run_config(s, precision, schedule)
    cs = s.to_c()
    needs_setup = bool(s.boxes or s.comps or s.tensors or s.disp or s.spheres or s.tensor3)
    setup = oracle.device_setup() if needs_setup else None
    return rb.run(rc, setup, C.cast(C.pointer(cs), C.c_void_p) if needs_setup else None)
