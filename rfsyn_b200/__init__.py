"""Python host mirror of the rfsyn-b200 C ABI (ctypes).

The product is the C-ABI library ``rfsyn_b200/lib/librfsyn_fdtd_b200.so``
(reference-compatible entry points in ``include/rfsyn_fdtd.h``, extensions in
``include/rfsyn_fdtd_b200.h``).  This module only binds it: every call goes
to the CUDA engine behind the library; there is no Python or CPU compute path.
Importing fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "librfsyn_fdtd_b200.so"

FIELD_EX, FIELD_EY, FIELD_EZ, FIELD_HX, FIELD_HY, FIELD_HZ = range(6)
SRC_SOFT, SRC_HARD = 0, 1
FP64, FP32 = 0, 1
SPLIT, FUSED = 0, 1
WAVE_GAUSSIAN_DERIV, WAVE_RICKER, WAVE_MOD_GAUSSIAN, WAVE_SAMPLES = range(4)

C0 = 299792458.0
EPS0 = 8.8541878128e-12
MU0 = 1.25663706212e-6


class FdtdSimConfig(C.Structure):
    """fdtd_sim_config_t (engine/fdtd/simulate.h:9-23)."""

    _fields_ = [
        ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
        ("dx", C.c_double), ("courant_safety", C.c_double), ("n_steps", C.c_size_t),
        ("npml", C.c_size_t),
        ("src_i", C.c_size_t), ("src_j", C.c_size_t), ("src_k", C.c_size_t),
        ("src_component", C.c_int), ("t0_over_dt", C.c_double), ("tau_over_dt", C.c_double),
        ("probe_i", C.c_size_t), ("probe_j", C.c_size_t), ("probe_k", C.c_size_t),
        ("probe_component", C.c_int),
    ]


class CpmlParams(C.Structure):
    """cpml_params_t (engine/fdtd/cpml.h:29-36)."""

    _fields_ = [("npml", C.c_size_t), ("m", C.c_double), ("ma", C.c_double),
                ("kappa_max", C.c_double), ("alpha_max", C.c_double), ("r0", C.c_double)]


class B200Source(C.Structure):
    _fields_ = [("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t), ("component", C.c_int),
                ("mode", C.c_int), ("amplitude", C.c_double), ("waveform", C.c_int),
                ("p0", C.c_double), ("p1", C.c_double), ("p2", C.c_double),
                ("samples", C.POINTER(C.c_double))]


class B200Probe(C.Structure):
    _fields_ = [("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t), ("component", C.c_int)]


class PlaneWave(C.Structure):
    """fdtd_b200_plane_wave_t."""

    _fields_ = [("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double), ("amplitude", C.c_double),
                ("waveform", C.c_int), ("p0", C.c_double), ("p1", C.c_double), ("p2", C.c_double),
                ("i0", C.c_size_t), ("i1", C.c_size_t), ("j0", C.c_size_t), ("j1", C.c_size_t),
                ("k0", C.c_size_t), ("k1", C.c_size_t)]


class B200Plane(C.Structure):
    _fields_ = [("axis", C.c_int), ("index", C.c_size_t), ("component", C.c_int)]


class B200Config(C.Structure):
    _fields_ = [
        ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t),
        ("dx", C.c_double), ("courant_safety", C.c_double), ("n_steps", C.c_size_t),
        ("periodic_axes", C.c_uint), ("cpml", CpmlParams), ("precision", C.c_int), ("schedule", C.c_int),
        ("n_sources", C.c_size_t), ("sources", C.POINTER(B200Source)), ("source_time_offset_steps", C.c_double),
        ("n_probes", C.c_size_t), ("probes", C.POINTER(B200Probe)),
        ("n_freqs", C.c_size_t), ("freqs_hz", C.POINTER(C.c_double)), ("dft_time_offset_steps", C.c_double),
        ("plane_wave", C.POINTER(PlaneWave)),
        ("n_planes", C.c_size_t), ("planes", C.POINTER(B200Plane)),
    ]


class B200Result(C.Structure):
    _fields_ = [("probe_td", C.POINTER(C.c_double)), ("dft_re", C.POINTER(C.c_double)),
                ("dft_im", C.POINTER(C.c_double)), ("sample_rate_hz", C.c_double), ("device_ms", C.c_double)]


class Dispersive(C.Structure):
    """fdtd_b200_dispersive_t."""

    _fields_ = [("eps_inf", C.c_double), ("sigma", C.c_double), ("n_poles", C.c_int), ("kind", C.c_int * 2),
                ("delta_eps", C.c_double * 2), ("tau", C.c_double * 2), ("omega_p", C.c_double * 2),
                ("gamma", C.c_double * 2)]


class Sphere(C.Structure):
    """fdtd_b200_sphere_t."""

    _fields_ = [("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double), ("radius", C.c_double),
                ("eps_r", C.c_double), ("sigma", C.c_double), ("model", C.POINTER(Dispersive))]


class SimInfo(C.Structure):
    _fields_ = [("cells", C.c_size_t), ("list_cells", C.c_size_t), ("dispersive", C.c_size_t),
                ("slab_cell_axes", C.c_size_t), ("h2d_bytes", C.c_size_t), ("precision", C.c_int),
                ("schedule", C.c_int), ("tile_j", C.c_int), ("seg_len", C.c_int),
                ("ring_depth", C.c_int), ("tma", C.c_int), ("interior_items", C.c_int),
                ("edge_items", C.c_int), ("unified", C.c_int), ("interior_ring2", C.c_int), ("seg_edge", C.c_int)]


class Energy(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("electric_j", "magnetic_j", "total_j", "interior_j", "electric_prev_j",
                                           "cross_j", "modified_prev_j", "max_abs_e", "max_abs_h")] + \
               [("nonfinite", C.c_size_t)]


class BatchInfo(C.Structure):
    _fields_ = [("scenes", C.c_size_t), ("cells", C.c_size_t), ("list_cells", C.c_size_t),
                ("slab_cell_axes", C.c_size_t), ("tile_j", C.c_int), ("ring_depth", C.c_int), ("mode", C.c_int),
                ("seg_interior", C.c_int), ("seg_edge", C.c_int), ("items_interior", C.c_int),
                ("items_xslab", C.c_int), ("items_edge", C.c_int), ("launches_per_step", C.c_int),
                ("unified", C.c_int)]


SETUP_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)


def dispersive(eps_inf: float, sigma: float, poles) -> Dispersive:
    """poles: ("debye", delta_eps, tau) / ("lorentz", delta_eps, omega_p, gamma)."""
    d = Dispersive()
    d.eps_inf, d.sigma, d.n_poles = eps_inf, sigma, len(poles)
    for q, p in enumerate(poles):
        if p[0] == "debye":
            d.kind[q], d.delta_eps[q], d.tau[q] = 0, p[1], p[2]
        else:
            d.kind[q], d.delta_eps[q], d.omega_p[q], d.gamma[q] = 1, p[1], p[2], p[3]
    return d


class SphereSetup:
    """An fdtd_material_setup_fn that rasterises spheres through
    fdtd_b200_materials_add_spheres (keeps the ctypes objects alive)."""

    def __init__(self, spheres, smoothing: int = 1):
        lib = load()
        self._models = []
        self._arr = (Sphere * max(len(spheres), 1))()
        for q, (cx, cy, cz, r, eps, sig, model) in enumerate(spheres):
            sp = self._arr[q]
            sp.cx, sp.cy, sp.cz, sp.radius, sp.eps_r, sp.sigma = cx, cy, cz, r, eps, sig
            if model is not None:
                self._models.append(model)
                sp.model = C.pointer(model)
        n = len(spheres)

        def cb(grid, mat, ctx):
            return lib.fdtd_b200_materials_add_spheres(mat, grid, self._arr, n, smoothing)

        self.fn = SETUP_FN(cb)
        self.ptr = C.cast(self.fn, C.c_void_p)


class SceneSetup:
    """An fdtd_material_setup_fn that applies boxes (rfsyn's
    materials_set_box, in list order), spheres
    (fdtd_b200_materials_add_spheres), dispersive boxes
    (fdtd_b200_materials_set_dispersive_box) and last anisotropic slabs
    (fdtd_b200_materials_set_tensor3_slab, or with slab_smoothing
    fdtd_b200_materials_set_tensor3_slab_smoothed); keeps the ctypes objects
    alive.
    boxes: (i0, i1, j0, j1, k0, k1, eps_r, sigma) half-open cell ranges;
    slabs: (point[3], normal[3], thickness, eps_r[9]); disp_boxes:
    (i0, i1, j0, j1, k0, k1, Dispersive)."""

    def __init__(self, boxes=(), spheres=(), smoothing: int = 1, slabs=(), disp_boxes=(), slab_smoothing: int = 0):
        lib = load()
        set_slab = (lib.fdtd_b200_materials_set_tensor3_slab_smoothed if slab_smoothing
                    else lib.fdtd_b200_materials_set_tensor3_slab)
        self._spheres = SphereSetup(spheres, smoothing) if spheres else None
        boxes = list(boxes)
        self._slabs = [((C.c_double * 3)(*p), (C.c_double * 3)(*n), t, (C.c_double * 9)(*e))
                       for (p, n, t, e) in slabs]
        self._dboxes = list(disp_boxes)

        def cb(grid, mat, ctx):
            for (i0, i1, j0, j1, k0, k1, eps, sig) in boxes:
                if lib.materials_set_box(mat, grid, i0, i1, j0, j1, k0, k1, eps, sig) != 0:
                    return -1
            if self._spheres is not None and self._spheres.fn(grid, mat, ctx) != 0:
                return -1
            for (i0, i1, j0, j1, k0, k1, model) in self._dboxes:
                if lib.fdtd_b200_materials_set_dispersive_box(mat, grid, i0, i1, j0, j1, k0, k1,
                                                              C.byref(model)) != 0:
                    return -1
            for (p, n, t, e) in self._slabs:
                if set_slab(mat, grid, p, n, t, e) != 0:
                    return -1
            return 0

        self.fn = SETUP_FN(cb)
        self.ptr = C.cast(self.fn, C.c_void_p)

class Awgn(C.Structure):
    _fields_ = [("snr_db", C.c_float), ("seed", C.c_uint64), ("stream", C.c_uint64)]


class Heightmap(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t), ("dx", C.c_double),
                ("heights_m", C.POINTER(C.c_double)), ("column_materials", C.POINTER(C.c_uint8)),
                ("air_id", C.c_uint8)]


class Medium(C.Structure):
    _fields_ = [("eps_r", C.c_double), ("sigma", C.c_double)]


class HeightmapSetup:
    """An fdtd_material_setup_fn that maps a heightmap world onto the grid
    (fdtd_b200_materials_apply_heightmap).  heights: (nx, ny) metres;
    columns: (nx, ny) world material ids; media: [(eps_r, sigma)] per id.
    After the setup ran, `mixed` holds the number of cells cut by the
    surface."""

    def __init__(self, heights, columns, media, nz: int, dx: float, air_id: int = 0, smoothing: int = 1):
        lib = load()
        h = np.ascontiguousarray(heights, dtype=np.float64)
        ids = np.ascontiguousarray(columns, dtype=np.uint8)
        self._h, self._ids = h, ids
        self._media = (Medium * len(media))(*[Medium(e, s) for (e, s) in media])
        self.mixed = None
        mixed = C.c_size_t(0)

        def cb(grid, mat, ctx):
            hm = Heightmap(h.shape[0], h.shape[1], nz, dx, _dptr(h), ids.ctypes.data_as(C.POINTER(C.c_uint8)),
                           air_id)
            if lib.fdtd_b200_materials_apply_heightmap(mat, grid, C.byref(hm), self._media, len(media), smoothing,
                                                        C.byref(mixed)) != 0:
                return -1
            self.mixed = mixed.value
            return 0

        self.fn = SETUP_FN(cb)
        self.ptr = C.cast(self.fn, C.c_void_p)


_lib = None


def load() -> C.CDLL:
    """Loads the built library (raises if it is missing: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is not built; run `python -m rfsyn_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    P, D, S, I, V = C.c_void_p, C.c_double, C.c_size_t, C.c_int, None
    sig = {
        "fdtd_simulate_echo": (I, [C.POINTER(FdtdSimConfig), C.POINTER(D), C.POINTER(D)]),
        "fdtd_simulate_echo_with_setup": (I, [C.POINTER(FdtdSimConfig), C.POINTER(D), C.POINTER(D), P, P]),
        "fdtd_b200_run": (I, [C.POINTER(B200Config), P, P, C.POINTER(B200Result)]),
        "fdtd_b200_sim_create": (P, [C.POINTER(B200Config), P, P, P]),
        "fdtd_b200_sim_destroy": (V, [P]),
        "fdtd_b200_sim_reset": (I, [P]),
        "fdtd_b200_sim_advance": (I, [P, S]),
        "fdtd_b200_sim_synchronize": (I, [P]),
        "fdtd_b200_sim_advance_timed": (I, [P, S, C.POINTER(D)]),
        "fdtd_b200_sim_steps_done": (S, [P]),
        "fdtd_b200_sim_stream": (P, [P]),
        "fdtd_b200_sim_read_probes": (I, [P, C.POINTER(D)]),
        "fdtd_b200_sim_read_iq": (I, [P, S, C.POINTER(Awgn), C.POINTER(C.c_float)]),
        "fdtd_b200_iq_write": (I, [C.c_char_p, C.POINTER(C.c_float), S]),
        "fdtd_b200_sim_dft": (I, [P, C.POINTER(D), C.POINTER(D)]),
        "fdtd_b200_sim_read_field": (I, [P, I, C.POINTER(D)]),
        "fdtd_b200_sim_launches_per_step": (I, [P]),
        "fdtd_b200_last_error": (C.c_char_p, []),
        "fdtd_b200_launch_count": (C.c_ulonglong, []),
        "fdtd_b200_cached_bytes": (C.c_ulonglong, []),
        "fdtd_b200_release_cached_memory": (None, []),
        "fdtd_b200_apply_setting": (I, [C.c_char_p, C.c_char_p]),
        "fdtd_b200_get_setting": (I, [C.c_char_p, C.c_char_p, S]),
        "fdtd_b200_set_default_precision": (I, [I]),
        "fdtd_b200_set_default_schedule": (I, [I]),
        "fdtd_b200_version": (C.c_char_p, []),
        "cpml_default_params": (CpmlParams, [S]),
        "fdtd_b200_materials_add_spheres": (I, [P, P, C.POINTER(Sphere), S, I]),
        "fdtd_b200_materials_apply_heightmap": (I, [P, P, C.POINTER(Heightmap), C.POINTER(Medium), S, I,
                                                    C.POINTER(C.c_size_t)]),
        "materials_set_box": (I, [P, P, S, S, S, S, S, S, D, D]),
        "fdtd_b200_materials_set_dispersive_box": (I, [P, P, S, S, S, S, S, S, P]),
        "fdtd_b200_materials_set_tensor3_slab": (I, [P, P, C.POINTER(D), C.POINTER(D), D, C.POINTER(D)]),
        "fdtd_b200_materials_set_tensor3_slab_smoothed": (I, [P, P, C.POINTER(D), C.POINTER(D), D, C.POINTER(D)]),
        "fdtd_b200_subpixel_tensor3": (I, [D, C.POINTER(D), C.POINTER(D), C.POINTER(D), C.POINTER(D)]),
        "fdtd_b200_sim_info": (I, [P, C.POINTER(SimInfo)]),
        "fdtd_b200_sim_time_kernels": (I, [P, S, C.POINTER(D), C.POINTER(D)]),
        "fdtd_b200_sim_energy": (I, [P, I, I, C.POINTER(Energy)]),
        "fdtd_b200_batch_create": (P, [S, C.POINTER(B200Config), C.POINTER(P), C.POINTER(P), P]),
        "fdtd_b200_batch_destroy": (V, [P]),
        "fdtd_b200_batch_size": (S, [P]),
        "fdtd_b200_batch_reset": (I, [P]),
        "fdtd_b200_batch_advance": (I, [P, S]),
        "fdtd_b200_batch_advance_timed": (I, [P, S, C.POINTER(D)]),
        "fdtd_b200_batch_synchronize": (I, [P]),
        "fdtd_b200_batch_steps_done": (S, [P]),
        "fdtd_b200_batch_stream": (P, [P]),
        "fdtd_b200_batch_time_kernels": (I, [P, S, C.POINTER(D), C.POINTER(D)]),
        "fdtd_b200_batch_read_probes": (I, [P, S, C.POINTER(D)]),
        "fdtd_b200_batch_read_iq": (I, [P, S, S, C.POINTER(Awgn), C.POINTER(C.c_float)]),
        "fdtd_b200_batch_dft": (I, [P, S, C.POINTER(D), C.POINTER(D)]),
        "fdtd_b200_batch_info": (I, [P, C.POINTER(BatchInfo)]),
        "fdtd_b200_mlp_create": (P, [I, I, I, I, C.c_uint64]),
        "fdtd_b200_mlp_destroy": (V, [P]),
        "fdtd_b200_mlp_n_params": (S, [P]),
        "fdtd_b200_mlp_get_params": (I, [P, C.POINTER(C.c_float)]),
        "fdtd_b200_mlp_set_params": (I, [P, C.POINTER(C.c_float)]),
        "fdtd_b200_mlp_grad": (I, [P, C.POINTER(C.c_float), C.POINTER(C.c_float), I, C.POINTER(D),
                                   C.POINTER(C.c_float)]),
        "fdtd_b200_mlp_set_data": (I, [P, C.POINTER(C.c_float), C.POINTER(C.c_float), S]),
        "fdtd_b200_mlp_train": (I, [P, S, I, D, D, D, D, C.c_uint64, C.POINTER(D)]),
        "fdtd_b200_mlp_predict": (I, [P, C.POINTER(C.c_float), S, C.POINTER(C.c_float)]),
        "fdtd_b200_mlp_launch_count": (C.c_ulonglong, [P]),
        "fdtd_b200_mlp_tensor_core_launches": (C.c_ulonglong, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().fdtd_b200_last_error().decode()


def iq_write(path, iq: np.ndarray) -> None:
    """Writes complex64 samples as rfsyn's .iq file (interleaved float32 I/Q,
    fdtd_b200_iq_write)."""
    a = np.ascontiguousarray(iq, dtype=np.complex64)
    ptr = a.view(np.float32).ctypes.data_as(C.POINTER(C.c_float)) if a.size else None
    if load().fdtd_b200_iq_write(os.fsencode(path), ptr, a.size) != 0:
        raise OSError(f"could not write {path}: {last_error()}")


def cached_bytes() -> int:
    """Device memory the library keeps from destroyed simulations for reuse."""
    return int(load().fdtd_b200_cached_bytes())


def release_cached_memory() -> None:
    """Returns the library's cached device memory to the driver."""
    load().fdtd_b200_release_cached_memory()


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def simulate_echo(cfg: FdtdSimConfig, setup=None, context=None) -> tuple[int, np.ndarray, float]:
    """rfsyn's fdtd_simulate_echo[_with_setup] through the C ABI."""
    lib = load()
    out = np.zeros(max(cfg.n_steps, 1), dtype=np.float64)
    fs = C.c_double(0.0)
    if setup is None:
        rc = lib.fdtd_simulate_echo(C.byref(cfg), _dptr(out), C.byref(fs))
    else:
        rc = lib.fdtd_simulate_echo_with_setup(C.byref(cfg), _dptr(out), C.byref(fs), setup, context)
    return rc, out[: cfg.n_steps], fs.value


class RunConfig:
    """Builds an fdtd_b200_config_t and keeps the arrays it points to alive."""

    def __init__(self, nx, ny, nz, dx, n_steps, npml, *, courant=0.99, periodic=0, precision=FP64,
                 schedule=FUSED, cpml: CpmlParams | None = None, sources=(), probes=(), freqs=(),
                 source_time_offset=0.0, dft_time_offset=1.0, plane_wave: dict | None = None, planes=()):
        self.c = B200Config()
        c = self.c
        c.nx, c.ny, c.nz, c.dx, c.n_steps = nx, ny, nz, dx, n_steps
        c.courant_safety = courant
        c.periodic_axes = periodic
        c.cpml = cpml if cpml is not None else load().cpml_default_params(npml)
        if npml == 0:
            c.cpml.npml = 0
        c.precision, c.schedule = precision, schedule
        self._src = (B200Source * max(len(sources), 1))()
        self._samples = []
        for q, s in enumerate(sources):
            src = self._src[q]
            src.i, src.j, src.k = s["i"], s["j"], s["k"]
            src.component = s.get("component", FIELD_EZ)
            src.mode = s.get("mode", SRC_SOFT)
            src.amplitude = s.get("amplitude", 1.0)
            src.waveform = s.get("waveform", WAVE_GAUSSIAN_DERIV)
            src.p0, src.p1, src.p2 = s.get("p0", 0.0), s.get("p1", 1.0), s.get("p2", 1.0)
            if "samples" in s:
                arr = np.ascontiguousarray(s["samples"], dtype=np.float64)
                self._samples.append(arr)
                src.samples = _dptr(arr)
        c.n_sources = len(sources)
        c.sources = self._src
        c.source_time_offset_steps = source_time_offset
        self._probes = (B200Probe * max(len(probes), 1))()
        for q, p in enumerate(probes):
            self._probes[q].i, self._probes[q].j, self._probes[q].k = p["i"], p["j"], p["k"]
            self._probes[q].component = p.get("component", FIELD_EZ)
        c.n_probes = len(probes)
        c.probes = self._probes
        self._freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        c.n_freqs = len(self._freqs)
        c.freqs_hz = _dptr(self._freqs) if len(self._freqs) else None
        c.dft_time_offset_steps = dft_time_offset
        self._pw = None
        if plane_wave is not None:
            pw = PlaneWave()
            for name, _ in PlaneWave._fields_:
                setattr(pw, name, plane_wave.get(name, 0))
            self._pw = pw
            c.plane_wave = C.pointer(pw)
        self._planes = (B200Plane * max(len(planes), 1))()
        for q, pl in enumerate(planes):
            self._planes[q].axis, self._planes[q].index = pl["axis"], pl["index"]
            self._planes[q].component = pl.get("component", FIELD_EX)
        c.n_planes = len(planes)
        c.planes = self._planes

    @property
    def n_series(self) -> int:
        """Point probes, then plane probes."""
        return self.c.n_probes + self.c.n_planes


def run(rc: RunConfig, setup=None, context=None) -> dict:
    """fdtd_b200_run: one full run; returns probe series, DFT and GPU time."""
    lib = load()
    c = rc.c
    ns = rc.n_series
    td = np.zeros((max(ns, 1), c.n_steps))
    re = np.zeros((max(ns, 1), max(c.n_freqs, 1)))
    im = np.zeros_like(re)
    res = B200Result()
    res.probe_td = _dptr(td)
    res.dft_re = _dptr(re)
    res.dft_im = _dptr(im)
    status = lib.fdtd_b200_run(C.byref(c), setup, context, C.byref(res))
    if status != 0:
        raise RuntimeError(f"fdtd_b200_run failed: {last_error()}")
    return {"td": td[:ns], "dft": (re + 1j * im)[:ns, : c.n_freqs],
            "fs": res.sample_rate_hz, "device_ms": res.device_ms}


class Sim:
    """A resident session (fdtd_b200_sim_*)."""

    def __init__(self, rc: RunConfig, setup=None, context=None, stream: int | None = None):
        self.lib = load()
        self.rc = rc
        self.h = self.lib.fdtd_b200_sim_create(C.byref(rc.c), setup, context, stream)
        if not self.h:
            raise RuntimeError(f"fdtd_b200_sim_create failed: {last_error()}")

    def reset(self):
        if self.lib.fdtd_b200_sim_reset(self.h) != 0:
            raise RuntimeError(last_error())

    def advance(self, n: int):
        if self.lib.fdtd_b200_sim_advance(self.h, n) != 0:
            raise RuntimeError(last_error())

    def advance_timed(self, n: int) -> float:
        """Advances n steps and returns their GPU time in ms (CUDA events)."""
        ms = C.c_double(0.0)
        if self.lib.fdtd_b200_sim_advance_timed(self.h, n, C.byref(ms)) != 0:
            raise RuntimeError(last_error())
        return ms.value

    def synchronize(self):
        if self.lib.fdtd_b200_sim_synchronize(self.h) != 0:
            raise RuntimeError(last_error())

    @property
    def stream(self) -> int:
        return self.lib.fdtd_b200_sim_stream(self.h) or 0

    @property
    def launches_per_step(self) -> int:
        return self.lib.fdtd_b200_sim_launches_per_step(self.h)

    def info(self) -> SimInfo:
        si = SimInfo()
        if self.lib.fdtd_b200_sim_info(self.h, C.byref(si)) != 0:
            raise RuntimeError(last_error())
        return si

    def energy(self, x_lo: int = 0, x_hi: int | None = None) -> dict:
        """FP64 energy audit of the resident fields (fdtd_b200_sim_energy)."""
        en = Energy()
        hi = self.rc.c.nx if x_hi is None else x_hi
        if self.lib.fdtd_b200_sim_energy(self.h, x_lo, hi, C.byref(en)) != 0:
            raise RuntimeError(last_error())
        return {n: getattr(en, n) for n, _ in Energy._fields_}

    def time_kernels(self, n: int) -> tuple[float, float]:
        """Runs n steps kernel by kernel; returns (sweep_ms, other_ms)."""
        a, b = C.c_double(0), C.c_double(0)
        if self.lib.fdtd_b200_sim_time_kernels(self.h, n, C.byref(a), C.byref(b)) != 0:
            raise RuntimeError(last_error())
        return a.value, b.value

    def probes(self) -> np.ndarray:
        c, ns = self.rc.c, self.rc.n_series
        out = np.zeros((max(ns, 1), c.n_steps))
        if self.lib.fdtd_b200_sim_read_probes(self.h, _dptr(out)) != 0:
            raise RuntimeError(last_error())
        return out[:ns]

    def read_iq(self, probe: int, snr_db: float | None = None, seed: int = 0, stream: int = 0) -> np.ndarray:
        """The stage's complex64 signal of one probe, with rfsyn's AWGN when
        snr_db is given (fdtd_b200_sim_read_iq)."""
        n = self.rc.c.n_steps
        out = np.zeros(2 * n, dtype=np.float32)
        awgn = C.byref(Awgn(snr_db, seed, stream)) if snr_db is not None else None
        if self.lib.fdtd_b200_sim_read_iq(self.h, probe, awgn, out.ctypes.data_as(C.POINTER(C.c_float))) != 0:
            raise RuntimeError(last_error())
        return out.view(np.complex64)

    def dft(self) -> np.ndarray:
        c, ns = self.rc.c, self.rc.n_series
        re = np.zeros((max(ns, 1), max(c.n_freqs, 1)))
        im = np.zeros_like(re)
        if self.lib.fdtd_b200_sim_dft(self.h, _dptr(re), _dptr(im)) != 0:
            raise RuntimeError(last_error())
        return (re + 1j * im)[:ns, : c.n_freqs]

    def field(self, component: int) -> np.ndarray:
        c = self.rc.c
        out = np.zeros((c.nx + 1, c.ny + 1, c.nz + 1))
        if self.lib.fdtd_b200_sim_read_field(self.h, component, _dptr(out)) != 0:
            raise RuntimeError(last_error())
        return out

    def close(self):
        if self.h:
            self.lib.fdtd_b200_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dt_of(dx: float, courant: float = 0.99) -> float:
    return courant * (dx / (C0 * np.sqrt(3.0)))


class Batch:
    """Many independent scenes advanced together (fdtd_b200_batch_*).

    configs: RunConfig per scene (same precision and step count); setups /
    contexts: one setup pointer (or None) and context (or None) per scene."""

    def __init__(self, configs, setups=None, contexts=None, stream: int | None = None):
        self.lib = load()
        self.configs = list(configs)
        n = len(self.configs)
        self._cfgs = (B200Config * n)(*[rc.c for rc in self.configs])
        self._setups = (C.c_void_p * n)(*[(s if s is not None else None) for s in (setups or [None] * n)])
        self._ctx = (C.c_void_p * n)(*[(x if x is not None else None) for x in (contexts or [None] * n)])
        self.h = self.lib.fdtd_b200_batch_create(n, self._cfgs, self._setups, self._ctx, stream)
        if not self.h:
            raise RuntimeError(f"fdtd_b200_batch_create failed: {last_error()}")

    def __len__(self):
        return len(self.configs)

    def _ok(self, rc):
        if rc != 0:
            raise RuntimeError(last_error())

    def reset(self):
        self._ok(self.lib.fdtd_b200_batch_reset(self.h))

    def advance(self, n: int):
        self._ok(self.lib.fdtd_b200_batch_advance(self.h, n))

    def advance_timed(self, n: int) -> float:
        ms = C.c_double(0.0)
        self._ok(self.lib.fdtd_b200_batch_advance_timed(self.h, n, C.byref(ms)))
        return ms.value

    def synchronize(self):
        self._ok(self.lib.fdtd_b200_batch_synchronize(self.h))

    @property
    def stream(self) -> int:
        return self.lib.fdtd_b200_batch_stream(self.h) or 0

    def info(self) -> BatchInfo:
        bi = BatchInfo()
        self._ok(self.lib.fdtd_b200_batch_info(self.h, C.byref(bi)))
        return bi

    def time_kernels(self, n: int) -> tuple[float, float]:
        a, b = C.c_double(0), C.c_double(0)
        self._ok(self.lib.fdtd_b200_batch_time_kernels(self.h, n, C.byref(a), C.byref(b)))
        return a.value, b.value

    def probes(self, scene: int) -> np.ndarray:
        c = self.configs[scene].c
        out = np.zeros((max(c.n_probes, 1), c.n_steps))
        self._ok(self.lib.fdtd_b200_batch_read_probes(self.h, scene, _dptr(out)))
        return out[: c.n_probes]

    def read_iq(self, scene: int, probe: int, snr_db: float | None = None, seed: int = 0,
                stream: int = 0) -> np.ndarray:
        """complex64 stage signal of one probe of one scene, with rfsyn's AWGN
        when snr_db is given (fdtd_b200_batch_read_iq)."""
        n = self.configs[scene].c.n_steps
        out = np.zeros(2 * n, dtype=np.float32)
        awgn = C.byref(Awgn(snr_db, seed, stream)) if snr_db is not None else None
        self._ok(self.lib.fdtd_b200_batch_read_iq(self.h, scene, probe, awgn, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out.view(np.complex64)

    def dft(self, scene: int) -> np.ndarray:
        c = self.configs[scene].c
        re = np.zeros((max(c.n_probes, 1), max(c.n_freqs, 1)))
        im = np.zeros_like(re)
        self._ok(self.lib.fdtd_b200_batch_dft(self.h, scene, _dptr(re), _dptr(im)))
        return (re + 1j * im)[: c.n_probes, : c.n_freqs]

    def close(self):
        if self.h:
            self.lib.fdtd_b200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The surrogate's network on the GPU (fdtd_b200_mlp_*)."""

    def __init__(self, n_in: int, width: int, depth: int, n_out: int, seed: int = 0):
        self.lib = load()
        self.n_in, self.width, self.depth, self.n_out = n_in, width, depth, n_out
        self.h = self.lib.fdtd_b200_mlp_create(n_in, width, depth, n_out, seed)
        if not self.h:
            raise RuntimeError(f"fdtd_b200_mlp_create failed: {last_error()}")

    def _ok(self, rc):
        if rc != 0:
            raise RuntimeError(last_error())

    def tensor_core_launches(self) -> int:
        """Products run so far on the tcgen05 tensor cores."""
        return int(self.lib.fdtd_b200_mlp_tensor_core_launches(self.h))

    @property
    def n_params(self) -> int:
        return self.lib.fdtd_b200_mlp_n_params(self.h)

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        self._ok(self.lib.fdtd_b200_mlp_get_params(self.h, _fptr(out)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._ok(self.lib.fdtd_b200_mlp_set_params(self.h, _fptr(p)))

    def grad(self, X: np.ndarray, Y: np.ndarray) -> tuple[float, np.ndarray]:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double(0)
        self._ok(self.lib.fdtd_b200_mlp_grad(self.h, _fptr(X), _fptr(Y), X.shape[0], C.byref(loss), _fptr(g)))
        return loss.value, g

    def set_data(self, X: np.ndarray, Y: np.ndarray):
        self._X = np.ascontiguousarray(X, dtype=np.float32)
        self._Y = np.ascontiguousarray(Y, dtype=np.float32)
        self._ok(self.lib.fdtd_b200_mlp_set_data(self.h, _fptr(self._X), _fptr(self._Y), self._X.shape[0]))

    def train(self, steps: int, batch: int = 256, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
              eps: float = 1e-8, seed: int = 0) -> float:
        loss = C.c_double(0)
        self._ok(self.lib.fdtd_b200_mlp_train(self.h, steps, batch, lr, beta1, beta2, eps, seed, C.byref(loss)))
        return loss.value

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], self.n_out), dtype=np.float32)
        self._ok(self.lib.fdtd_b200_mlp_predict(self.h, _fptr(X), X.shape[0], _fptr(Y)))
        return Y

    def close(self):
        if self.h:
            self.lib.fdtd_b200_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
