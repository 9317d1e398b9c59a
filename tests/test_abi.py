"""The C ABI without a GPU: symbol exports, the host-side scene description
(rfsyn tests/materials_unit.c semantics), CPML profiles against rfsyn, and
the error conventions that trigger before any device work."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from tests.cases import simulate_unit_cfg

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_functions() -> list[str]:
    names = []
    for h in sorted(INCLUDE.glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^([A-Za-z_][\w \t\*]*?)\b([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;", text, flags=re.M):
            if m.group(1).strip().startswith(("typedef", "return")):
                continue
            names.append(m.group(2))
    return sorted(set(names))


def test_header_declares_the_rfsyn_entry_points():
    names = declared_functions()
    for must in ("fdtd_stage_create", "fdtd_simulate_echo", "fdtd_simulate_echo_with_setup", "fdtd_grid_create",
                 "cpml_create", "fdtd_update_h_cpml", "fdtd_update_e_cpml_materials", "materials_set_component_tensor",
                 "source_apply", "probe_dft_record", "signal_resize", "fdtd_b200_run", "fdtd_b200_sim_create"):
        assert must in names


def test_library_exports_every_declared_function():
    lib = rb.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def _api(lib):
    P, S, D, I = C.c_void_p, C.c_size_t, C.c_double, C.c_int
    lib.fdtd_grid_create.restype = P
    lib.fdtd_grid_create.argtypes = [S, S, S, D, D]
    lib.fdtd_grid_destroy.argtypes = [P]
    lib.fdtd_grid_set_periodic.argtypes = [P, C.c_uint]
    lib.materials_create.restype = P
    lib.materials_create.argtypes = [P]
    lib.materials_destroy.argtypes = [P]
    lib.materials_register.argtypes = [P, D, D, C.POINTER(C.c_uint8)]
    lib.materials_assign_box.argtypes = [P, P, S, S, S, S, S, S, C.c_uint8]
    lib.materials_set_box.argtypes = [P, P, S, S, S, S, S, S, D, D]
    lib.materials_set_component.argtypes = [P, P, I, S, S, S, D, D]
    lib.materials_clear_component.argtypes = [P, P, I, S, S, S]
    lib.materials_get_coefficients.argtypes = [P, P, I, S, S, S, P]
    lib.materials_set_component_tensor.argtypes = [P, P, I, S, S, S, D, D, D]
    lib.materials_clear_component_tensor.argtypes = [P, P, I, S, S, S]
    lib.materials_get_tensor.argtypes = [P, P, I, S, S, S, P]
    lib.cpml_create.restype = P
    lib.cpml_create.argtypes = [P, rb.CpmlParams]
    lib.cpml_destroy.argtypes = [P]
    lib.cpml_default_params.restype = rb.CpmlParams
    lib.cpml_default_params.argtypes = [S]
    return lib


class Coeff(C.Structure):
    _fields_ = [("Ca", C.c_double), ("Cb", C.c_double)]


class Tensor(C.Structure):
    _fields_ = [("m11", C.c_double), ("m12", C.c_double), ("m22", C.c_double), ("scale", C.c_double)]


def _materials_script(lib):
    """rfsyn tests/materials_unit.c (host part) plus tensor / box clearing;
    returns every observable as a list so two libraries can be compared."""
    lib = _api(lib)
    out = []
    g = lib.fdtd_grid_create(12, 12, 12, 1e-3, 0.99)
    m = lib.materials_create(g)
    co = Coeff()
    tid = C.c_uint8()
    t = Tensor()
    out.append(lib.materials_get_coefficients(m, g, 0, 6, 6, 6, C.byref(co)))
    out += [co.Ca, co.Cb]
    out.append(lib.materials_register(m, 4.0, 0.0, C.byref(tid)))
    out.append(tid.value)
    out.append(lib.materials_register(m, 4.0, 0.0, C.byref(tid)))
    out.append(tid.value)
    out.append(lib.materials_assign_box(m, g, 5, 8, 5, 8, 5, 8, tid.value))
    for comp, ijk in ((1, (6, 6, 6)), (0, (4, 6, 6))):
        out.append(lib.materials_get_coefficients(m, g, comp, *ijk, C.byref(co)))
        out += [co.Ca, co.Cb]
    out.append(lib.materials_set_component(m, g, 0, 6, 6, 6, 9.0, 0.1))
    out.append(lib.materials_set_component(m, g, 2, 6, 6, 6, 16.0, 0.0))
    for comp in range(3):
        out.append(lib.materials_get_coefficients(m, g, comp, 6, 6, 6, C.byref(co)))
        out += [co.Ca, co.Cb]
    out.append(lib.materials_clear_component(m, g, 0, 6, 6, 6))
    out.append(lib.materials_get_coefficients(m, g, 0, 6, 6, 6, C.byref(co)))
    out += [co.Ca, co.Cb]
    out.append(lib.materials_set_box(m, g, 6, 7, 6, 7, 6, 7, 1.0, 0.0))
    out.append(lib.materials_get_coefficients(m, g, 2, 6, 6, 6, C.byref(co)))
    out += [co.Ca, co.Cb]
    # error conventions
    out.append(lib.materials_set_box(m, g, 0, 14, 0, 1, 0, 1, 4.0, 0.0))
    out.append(lib.materials_register(m, float("nan"), 0.0, C.byref(tid)))
    out.append(lib.materials_register(m, 4.0, -1.0, C.byref(tid)))
    out.append(lib.materials_register(m, 0.5, 0.0, C.byref(tid)))
    out.append(lib.materials_set_component(m, g, 3, 6, 6, 6, 4.0, 0.0))
    out.append(lib.materials_set_component(m, g, 0, 12, 6, 6, 4.0, 0.0))
    out.append(lib.materials_set_component(m, g, 1, 12, 6, 6, 4.0, 0.0))
    out.append(lib.materials_get_coefficients(m, g, 0, 6, 6, 6, None))
    # tensors: margins, SPD test, precedence, box clearing
    out.append(lib.materials_set_component_tensor(m, g, 0, 3, 3, 3, 0.3, 0.05, 0.25))
    out.append(lib.materials_set_component_tensor(m, g, 0, 0, 3, 3, 0.3, 0.05, 0.25))
    out.append(lib.materials_set_component_tensor(m, g, 0, 3, 11, 3, 0.3, 0.05, 0.25))
    out.append(lib.materials_set_component_tensor(m, g, 0, 3, 3, 3, 0.3, 0.5, 0.25))
    out.append(lib.materials_set_component_tensor(m, g, 2, 3, 3, 3, 0.3, 0.05, 0.25))
    out.append(lib.materials_get_tensor(m, g, 0, 3, 3, 3, C.byref(t)))
    out += [t.m11, t.m12, t.m22, t.scale]
    out.append(lib.materials_get_tensor(m, g, 1, 3, 3, 3, C.byref(t)))
    out.append(lib.materials_assign_box(m, g, 3, 4, 3, 4, 3, 4, 0))
    out.append(lib.materials_get_tensor(m, g, 0, 3, 3, 3, C.byref(t)))
    out.append(lib.materials_set_component_tensor(m, g, 1, 4, 4, 4, 0.2, 0.01, 0.3))
    out.append(lib.materials_clear_component_tensor(m, g, 1, 4, 4, 4))
    out.append(lib.materials_get_tensor(m, g, 1, 4, 4, 4, C.byref(t)))
    # material table limit (256 entries, vacuum included)
    codes = [lib.materials_register(m, 1.0 + q * 0.01, 0.0, C.byref(tid)) for q in range(300)]
    out.append(codes.count(0))
    out.append(codes.count(-1))
    # periodic: component validity drops the duplicate endpoint
    gp = lib.fdtd_grid_create(6, 6, 6, 1e-3, 0.99)
    lib.fdtd_grid_set_periodic(gp, 5)
    mp = lib.materials_create(gp)
    out.append(lib.materials_set_component(mp, gp, 1, 6, 0, 0, 2.0, 0.0))
    out.append(lib.materials_set_component(mp, gp, 0, 5, 6, 0, 2.0, 0.0))
    out.append(lib.materials_set_box(mp, gp, 6, 7, 0, 1, 0, 1, 2.0, 0.0))
    out.append(lib.materials_set_box(mp, gp, 0, 7, 0, 7, 0, 7, 2.0, 0.0))
    lib.materials_destroy(mp)
    lib.fdtd_grid_destroy(gp)
    lib.materials_destroy(m)
    lib.fdtd_grid_destroy(g)
    return out


def test_materials_host_semantics_match_rfsyn():
    ours = _materials_script(rb.load())
    # rfsyn tests/materials_unit.c expectations
    assert ours[0] == 0 and ours[1] == 1.0
    eps0 = 8.8541878128e-12
    dt = rb.dt_of(1e-3)
    assert abs(ours[2] - dt / (eps0 * 1e-3)) <= 1e-12 * ours[2]
    if oracle.ref_available():
        theirs = _materials_script(C.CDLL(str(oracle.REF_LIB)))
        assert ours == theirs


@pytest.mark.parametrize("per", range(8))
def test_cpml_profiles_match_rfsyn(per):
    if not oracle.ref_available():
        pytest.skip("rfsyn sources not built here")
    libs = [_api(rb.load()), _api(C.CDLL(str(oracle.REF_LIB)))]
    arrays = []
    for lib in libs:
        g = lib.fdtd_grid_create(23, 17, 30, 0.5e-3, 0.99)
        lib.fdtd_grid_set_periodic(g, per)
        p = lib.cpml_create(g, rb.CpmlParams(6, 3.0, 1.0, 5.0, 0.05, 1e-6))
        assert p
        # struct cpml: npml, dx, then 18 profile pointers (cpml.h:7-25)
        ptrs = C.cast(p, C.POINTER(C.c_void_p))
        lens = []
        for ax_n in (23, 17, 30):
            lens += [ax_n + 1] * 3
        for ax_n in (23, 17, 30):
            lens += [ax_n] * 3
        vals = []
        for q, n in enumerate(lens):
            arr = C.cast(ptrs[2 + q], C.POINTER(C.c_double))
            vals.append(np.ctypeslib.as_array(arr, shape=(n,)).copy())
        arrays.append(vals)
        lib.cpml_destroy(p)
        lib.fdtd_grid_destroy(g)
    for a, b in zip(*arrays):
        assert np.array_equal(a, b)


def test_cpml_rejects_what_rfsyn_rejects():
    lib = _api(rb.load())
    g = lib.fdtd_grid_create(10, 10, 10, 1e-3, 0.99)
    bad = [rb.CpmlParams(0, 3, 1, 7, 0.05, 1e-6), rb.CpmlParams(5, 3, 1, 7, 0.05, 1e-6),
           rb.CpmlParams(2, 0, 1, 7, 0.05, 1e-6), rb.CpmlParams(2, 3, -1, 7, 0.05, 1e-6),
           rb.CpmlParams(2, 3, 1, 0.5, 0.05, 1e-6), rb.CpmlParams(2, 3, 1, 7, -0.1, 1e-6),
           rb.CpmlParams(2, 3, 1, 7, 0.05, 1.0), rb.CpmlParams(2, 3, 1, 7, 0.05, float("nan"))]
    for p in bad:
        assert not lib.cpml_create(g, p)
    assert lib.cpml_create(g, rb.CpmlParams(4, 3, 1, 7, 0.05, 1e-6))
    lib.fdtd_grid_destroy(g)


def test_grid_create_rejections():
    lib = _api(rb.load())
    for args in ((0, 4, 4, 1e-3, 0.99), (4, 4, 4, 0.0, 0.99), (4, 4, 4, 1e-3, 0.0), (4, 4, 4, 1e-3, 1.5),
                 (4, 4, 4, float("inf"), 0.99)):
        assert not lib.fdtd_grid_create(*args)
    g = lib.fdtd_grid_create(4, 5, 6, 1e-3, 1.0)
    assert g
    assert lib.fdtd_grid_set_periodic(g, 8) == -1
    assert lib.fdtd_grid_set_periodic(None, 1) == -1
    lib.fdtd_grid_destroy(g)


def test_simulate_error_returns_before_device_work():
    # rfsyn tests/simulate_unit.c:107-131
    cfg = simulate_unit_cfg()
    bad = simulate_unit_cfg()
    bad.n_steps = 0
    assert rb.simulate_echo(bad)[0] == -1
    bad = simulate_unit_cfg()
    bad.probe_i = cfg.nx + 1
    assert rb.simulate_echo(bad)[0] == -1
    bad = simulate_unit_cfg()
    bad.src_k = cfg.nz + 1
    assert rb.simulate_echo(bad)[0] == -1
    lib = rb.load()
    out = np.zeros(4)
    assert lib.fdtd_simulate_echo(None, out.ctypes.data_as(C.POINTER(C.c_double)), None) == -1
    assert lib.fdtd_simulate_echo(C.byref(cfg), None, None) == -1


def test_stage_create_null_and_copy():
    lib = rb.load()

    class Transform(C.Structure):
        _fields_ = [("apply", C.c_void_p), ("destroy", C.c_void_p), ("ctx", C.c_void_p)]

    lib.fdtd_stage_create.restype = Transform
    lib.fdtd_stage_create.argtypes = [C.c_void_p]
    t = lib.fdtd_stage_create(None)
    assert not t.apply and not t.destroy and not t.ctx
    cfg = simulate_unit_cfg()
    t = lib.fdtd_stage_create(C.byref(cfg))
    assert t.apply and t.destroy and t.ctx
    DESTROY = C.CFUNCTYPE(None, C.c_void_p)
    DESTROY(t.destroy)(t.ctx)


def test_signal_resize_semantics():
    lib = rb.load()

    class Signal(C.Structure):
        _fields_ = [("samples", C.c_void_p), ("n_samples", C.c_size_t), ("sample_rate_hz", C.c_double),
                    ("center_freq_hz", C.c_double), ("metadata", C.c_void_p), ("meta_copy", C.c_void_p),
                    ("meta_free", C.c_void_p)]

    lib.signal_create.restype = C.POINTER(Signal)
    lib.signal_create.argtypes = [C.c_size_t, C.c_double, C.c_double]
    lib.signal_resize.argtypes = [C.POINTER(Signal), C.c_size_t]
    lib.signal_destroy.argtypes = [C.POINTER(Signal)]
    s = lib.signal_create(3, 1.0, 2.0)
    assert s.contents.n_samples == 3
    assert lib.signal_resize(s, 10) == 0 and s.contents.n_samples == 10
    vals = np.ctypeslib.as_array(C.cast(s.contents.samples, C.POINTER(C.c_float)), shape=(20,))
    assert np.all(vals == 0)
    assert lib.signal_resize(None, 4) == -1
    lib.signal_destroy(s)
