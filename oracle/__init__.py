"""TEST INFRASTRUCTURE: Python bindings of the FDTD oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, always as the checker.  Three CPU/GPU implementations of one
scene description (oracle/scene.h) are bound here:

* ``run_oracle``   -- the CPU restatement (oracle/fdtd_oracle.c, FP64),
* ``run_ref``      -- rfsyn itself built from its sources (oracle/_ref),
                      when that build exists,
* ``run_stepwise`` -- the same driver over librfsyn_fdtd_b200.so, i.e. the
                      GPU behind rfsyn's step-wise fdtd_update_* calls,
and ``device_setup`` gives the scene as an fdtd_material_setup_fn for the
product's device time loop.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# rfsyn's source tree, read (never written) only to compile rfsyn and its
# validators for the checker; the Makefile takes the same directory as REF
REFERENCE = Path(os.environ.get("RFSYN_REFERENCE_DIR", "/root/reference"))
ORACLE_LIB = HERE / "lib" / "liboracle.so"
DRIVER_LIB = HERE / "lib" / "libscene_driver_b200.so"
REF_LIB = HERE / "_ref" / "librfsyn_ref.so"


class ScnBox(C.Structure):
    _fields_ = [("i0", C.c_size_t), ("i1", C.c_size_t), ("j0", C.c_size_t), ("j1", C.c_size_t),
                ("k0", C.c_size_t), ("k1", C.c_size_t), ("eps_r", C.c_double), ("sigma", C.c_double)]


class ScnComp(C.Structure):
    _fields_ = [("comp", C.c_int), ("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t),
                ("eps_r", C.c_double), ("sigma", C.c_double)]


class ScnTensor(C.Structure):
    _fields_ = [("comp", C.c_int), ("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t),
                ("m11", C.c_double), ("m12", C.c_double), ("m22", C.c_double)]


class ScnSource(C.Structure):
    _fields_ = [("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t), ("comp", C.c_int), ("mode", C.c_int),
                ("amplitude", C.c_double), ("waveform", C.c_int), ("p0", C.c_double), ("p1", C.c_double),
                ("p2", C.c_double)]


class ScnProbe(C.Structure):
    _fields_ = [("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t), ("comp", C.c_int)]


class ScnDisp(C.Structure):
    _fields_ = [("comp", C.c_int), ("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t),
                ("eps_inf", C.c_double), ("sigma", C.c_double), ("npoles", C.c_int), ("kind", C.c_int * 2),
                ("delta_eps", C.c_double * 2), ("tau", C.c_double * 2), ("omega_p", C.c_double * 2),
                ("gamma", C.c_double * 2)]


class ScnSphere(C.Structure):
    _fields_ = [("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double), ("radius", C.c_double),
                ("eps_r", C.c_double), ("sigma", C.c_double), ("disp", C.c_int)]


MODEL_ONLY = (1 << 64) - 1  # i of a dispersive entry used only as a sphere material


def disp_entry(comp, i, j, k, eps_inf, sigma, poles):
    """poles: list of ("debye", delta_eps, tau) / ("lorentz", delta_eps, omega_p, gamma)."""
    kind, de, tau, wp, gm = [0, 0], [0.0, 0.0], [0.0, 0.0], [0.0, 0.0], [0.0, 0.0]
    for q, p in enumerate(poles):
        if p[0] == "debye":
            kind[q], de[q], tau[q] = 0, p[1], p[2]
        else:
            kind[q], de[q], wp[q], gm[q] = 1, p[1], p[2], p[3]
    return (comp, i, j, k, eps_inf, sigma, len(poles), tuple(kind), tuple(de), tuple(tau), tuple(wp), tuple(gm))


class ScnPlane(C.Structure):
    _fields_ = [("axis", C.c_int), ("index", C.c_size_t), ("comp", C.c_int)]


class ScnTensor3(C.Structure):
    _fields_ = [("comp", C.c_int), ("i", C.c_size_t), ("j", C.c_size_t), ("k", C.c_size_t),
                ("m", C.c_double * 3), ("sigma", C.c_double)]


class ScnPlaneWave(C.Structure):
    _fields_ = [("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double), ("amplitude", C.c_double),
                ("waveform", C.c_int), ("p0", C.c_double), ("p1", C.c_double), ("p2", C.c_double),
                ("i0", C.c_size_t), ("i1", C.c_size_t), ("j0", C.c_size_t), ("j1", C.c_size_t),
                ("k0", C.c_size_t), ("k1", C.c_size_t)]


class ScnScene(C.Structure):
    _fields_ = [
        ("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t), ("dx", C.c_double), ("courant", C.c_double),
        ("n_steps", C.c_size_t), ("periodic", C.c_uint), ("npml", C.c_size_t),
        ("m", C.c_double), ("ma", C.c_double), ("kappa_max", C.c_double), ("alpha_max", C.c_double),
        ("r0", C.c_double),
        ("n_boxes", C.c_size_t), ("boxes", C.POINTER(ScnBox)),
        ("n_comps", C.c_size_t), ("comps", C.POINTER(ScnComp)),
        ("n_tensors", C.c_size_t), ("tensors", C.POINTER(ScnTensor)),
        ("n_disp", C.c_size_t), ("disp", C.POINTER(ScnDisp)),
        ("n_spheres", C.c_size_t), ("spheres", C.POINTER(ScnSphere)),
        ("smoothing", C.c_int),
        ("n_sources", C.c_size_t), ("sources", C.POINTER(ScnSource)),
        ("n_probes", C.c_size_t), ("probes", C.POINTER(ScnProbe)),
        ("n_freqs", C.c_size_t), ("freqs", C.POINTER(C.c_double)),
        ("src_t_offset", C.c_double), ("dft_t_offset", C.c_double),
        ("n_tensor3", C.c_size_t), ("tensor3", C.POINTER(ScnTensor3)),
        ("plane_wave", C.POINTER(ScnPlaneWave)),
        ("n_planes", C.c_size_t), ("planes", C.POINTER(ScnPlane)),
    ]


@dataclass
class Scene:
    """A test case; lists hold tuples in the field order of the C structs."""

    nx: int
    ny: int
    nz: int
    dx: float = 1e-3
    courant: float = 0.99
    n_steps: int = 100
    periodic: int = 0
    npml: int = 0
    m: float = 3.0
    ma: float = 1.0
    kappa_max: float = 7.0
    alpha_max: float = 0.05
    r0: float = 1e-6
    boxes: list = field(default_factory=list)      # (i0,i1,j0,j1,k0,k1,eps,sigma)
    comps: list = field(default_factory=list)      # (comp,i,j,k,eps,sigma)
    tensors: list = field(default_factory=list)    # (comp,i,j,k,m11,m12,m22)
    disp: list = field(default_factory=list)       # disp_entry(...) tuples
    spheres: list = field(default_factory=list)    # (cx,cy,cz,r,eps,sigma,disp_index or -1)
    smoothing: int = 1
    sources: list = field(default_factory=list)    # (i,j,k,comp,mode,amp,waveform,p0,p1,p2)
    probes: list = field(default_factory=list)     # (i,j,k,comp)
    planes: list = field(default_factory=list)     # (axis,index,comp) plane probes, series after the probes
    freqs: list = field(default_factory=list)
    src_t_offset: float = 0.0
    dft_t_offset: float = 1.0
    tensor3: list = field(default_factory=list)    # (comp,i,j,k,(m0,m1,m2)[,sigma]) rows of eps_r^-1, applied last
    plane_wave: dict | None = None                  # ScnPlaneWave fields by name

    @property
    def dt(self) -> float:
        return self.courant * (self.dx / (299792458.0 * np.sqrt(3.0)))

    def to_c(self) -> ScnScene:
        """Returns the C struct; the arrays stay alive as attributes of it."""
        s = ScnScene()
        for name in ("nx", "ny", "nz", "dx", "courant", "n_steps", "periodic", "npml", "m", "ma", "kappa_max",
                     "alpha_max", "r0", "src_t_offset", "dft_t_offset", "smoothing"):
            setattr(s, name, getattr(self, name))
        keep = []

        def arr(typ, rows):
            a = (typ * max(len(rows), 1))(*[typ(*r) for r in rows])
            keep.append(a)
            return len(rows), a

        s.n_boxes, s.boxes = arr(ScnBox, self.boxes)
        s.n_comps, s.comps = arr(ScnComp, self.comps)
        s.n_tensors, s.tensors = arr(ScnTensor, self.tensors)
        drows = []
        for d in self.disp:
            comp, i, j, k, ei, sg, npl, kind, de, tau, wp, gm = d
            drows.append((comp, i, j, k, ei, sg, npl, (C.c_int * 2)(*kind), (C.c_double * 2)(*de),
                          (C.c_double * 2)(*tau), (C.c_double * 2)(*wp), (C.c_double * 2)(*gm)))
        s.n_disp, s.disp = arr(ScnDisp, drows)
        s.n_spheres, s.spheres = arr(ScnSphere, self.spheres)
        s.n_tensor3, s.tensor3 = arr(ScnTensor3, [(t[0], t[1], t[2], t[3], (C.c_double * 3)(*t[4]),
                                                   t[5] if len(t) > 5 else 0.0) for t in self.tensor3])
        if self.plane_wave is not None:
            pw = ScnPlaneWave()
            for name, _ in ScnPlaneWave._fields_:
                setattr(pw, name, self.plane_wave.get(name, 0))
            keep.append(pw)
            s.plane_wave = C.pointer(pw)
        s.n_sources, s.sources = arr(ScnSource, self.sources)
        s.n_probes, s.probes = arr(ScnProbe, self.probes)
        s.n_planes, s.planes = arr(ScnPlane, self.planes)
        f = (C.c_double * max(len(self.freqs), 1))(*self.freqs)
        keep.append(f)
        s.n_freqs, s.freqs = len(self.freqs), f
        s._keep = keep
        return s


def build(ref: bool = True) -> None:
    """Builds liboracle.so (and rfsyn's own sources into _ref when present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if ref and (REFERENCE / "engine/fdtd/grid.c").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REFERENCE}", "ref"], check=True)


def build_driver() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "driver"], check=True)
    if (REFERENCE / "engine/fdtd/grid.c").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REFERENCE}", "validators"], check=True)


_libs: dict[str, C.CDLL] = {}


def _load(path: Path, prefix: str) -> C.CDLL:
    key = str(path)
    if key not in _libs:
        if not path.exists():
            raise FileNotFoundError(path)
        lib = C.CDLL(key)
        run = getattr(lib, f"{prefix}_run")
        run.restype = C.c_int
        run.argtypes = [C.POINTER(ScnScene), C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        runf = getattr(lib, f"{prefix}_run_fields")
        runf.restype = C.c_int
        runf.argtypes = [C.POINTER(ScnScene), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _libs[key] = lib
    return _libs[key]


def ref_available() -> bool:
    return REF_LIB.exists()


def _run(lib: C.CDLL, prefix: str, scene: Scene):
    s = scene.to_c()
    npb, nf, nt = len(scene.probes) + len(scene.planes), len(scene.freqs), scene.n_steps
    td = np.zeros(max(npb * nt, 1))
    re = np.zeros(max(npb * nf, 1))
    im = np.zeros(max(npb * nf, 1))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rc = getattr(lib, f"{prefix}_run")(C.byref(s), dp(td), dp(re), dp(im))
    if rc != 0:
        raise RuntimeError(f"{prefix}_run failed")
    return {"td": td[: npb * nt].reshape(npb, nt), "dft": (re + 1j * im)[: npb * nf].reshape(npb, nf)}


def _run_fields(lib, prefix, scene: Scene, initial: np.ndarray | None):
    s = scene.to_c()
    total = (scene.nx + 1) * (scene.ny + 1) * (scene.nz + 1)
    out = np.zeros(6 * total)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ini = None if initial is None else np.ascontiguousarray(initial, dtype=np.float64).reshape(-1)
    rc = getattr(lib, f"{prefix}_run_fields")(C.byref(s), None if ini is None else dp(ini), dp(out))
    if rc != 0:
        raise RuntimeError(f"{prefix}_run_fields failed")
    return out.reshape(6, scene.nx + 1, scene.ny + 1, scene.nz + 1)


def run_oracle(scene: Scene):
    return _run(_load(ORACLE_LIB, "orc"), "orc", scene)


def run_ref(scene: Scene):
    return _run(_load(REF_LIB, "scn"), "scn", scene)


def run_stepwise(scene: Scene):
    return _run(_load(DRIVER_LIB, "scn"), "scn", scene)


def fields_oracle(scene: Scene, initial=None):
    return _run_fields(_load(ORACLE_LIB, "orc"), "orc", scene, initial)


def fields_ref(scene: Scene, initial=None):
    return _run_fields(_load(REF_LIB, "scn"), "scn", scene, initial)


def fields_stepwise(scene: Scene, initial=None):
    return _run_fields(_load(DRIVER_LIB, "scn"), "scn", scene, initial)


def energy_oracle(scene: Scene, x_lo: int = 0, x_hi: int | None = None) -> dict:
    """The oracle's energy audit after the scene's n_steps (orc_energy)."""
    lib = _load(ORACLE_LIB, "orc")
    f = lib.orc_energy
    f.restype = C.c_int
    f.argtypes = [C.POINTER(ScnScene), C.c_int, C.c_int, C.POINTER(C.c_double)]
    q = (C.c_double * 9)()
    s = scene.to_c()
    if f(C.byref(s), x_lo, scene.nx if x_hi is None else x_hi, q) != 0:
        raise RuntimeError("orc_energy failed")
    names = ("electric_j", "magnetic_j", "interior_e_j", "interior_h_j", "electric_prev_j", "cross_j",
             "max_abs_e", "max_abs_h", "nonfinite")
    return dict(zip(names, list(q)))


def device_setup():
    """scn_setup of the product-linked driver as a C function pointer."""
    lib = _load(DRIVER_LIB, "scn")
    return C.cast(lib.scn_setup, C.c_void_p)


def ref_simulate_echo(cfg) -> tuple[int, np.ndarray, float]:
    """rfsyn's own fdtd_simulate_echo (oracle/_ref)."""
    lib = _load(REF_LIB, "scn")
    f = lib.fdtd_simulate_echo
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    out = np.zeros(max(cfg.n_steps, 1))
    fs = C.c_double(0)
    rc = f(C.byref(cfg), out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(fs))
    return rc, out[: cfg.n_steps], fs.value
