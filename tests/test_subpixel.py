"""Subpixel smoothing helpers, on the host (no GPU).

rfsyn's 2-D helpers (engine/fdtd/subpixel_te.h) are exported by the product
library: rfsyn's own unit test (tests/subpixel_te_unit.c), compiled unmodified
and linked against the product, prints what it prints against rfsyn; the
known answers of that file's edge-fraction / tensor block (:572-631, which
its main() never calls) hold too, except two edge cases whose expectations
contradict the geometry (see the test); and on random inputs every helper
agrees with rfsyn's compiled code -- the edge fraction only where the
rectangle is unrotated: for a rotated one rfsyn's direction terms
(engine/fdtd/subpixel_te.c:56-58) measure an edge turned by twice the angle
(axis 1) or mirrored (axis 2), no rfsyn code calls the function, and the
product returns the geometric share, checked here by sampling.  The 3-D mix
fdtd_b200_subpixel_tensor3 is pinned
to rfsyn's 2x2 rule in the z-invariant limit, to the closed isotropic form,
and to the oracle's independent numpy restatement of Kottke et al.'s tau
average for anisotropic media."""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle.subpixel_oracle import isotropic_minv, smoothed_minv

ROOT = Path(__file__).resolve().parents[1]
D = C.c_double
PD = C.POINTER(C.c_double)


class Rect(C.Structure):
    _fields_ = [("center_x", D), ("center_y", D), ("size_u", D), ("size_v", D), ("angle_rad", D)]


def _bind(lib):
    lib.subpixel_te_rectangle_fraction.argtypes = [C.POINTER(Rect), D, D, D, D, PD]
    lib.subpixel_te_rectangle_edge_fraction.argtypes = [C.POINTER(Rect), D, D, C.c_int, D, PD]
    lib.subpixel_te_mix_epsilon_harmonic.argtypes = [D, D, D, PD]
    lib.subpixel_te_mix_epsilon.argtypes = [D, D, D, PD]
    lib.subpixel_te_rectangle_epsilon.argtypes = [C.POINTER(Rect), D, D, D, D, D, D, PD, PD]
    lib.subpixel_te_mix_epsilon_tensor.argtypes = [D, D, D, D, PD, PD, PD]
    for name in ("subpixel_te_rectangle_fraction", "subpixel_te_rectangle_edge_fraction",
                 "subpixel_te_mix_epsilon_harmonic", "subpixel_te_mix_epsilon", "subpixel_te_rectangle_epsilon",
                 "subpixel_te_mix_epsilon_tensor"):
        getattr(lib, name).restype = C.c_int
    return lib


@pytest.fixture(scope="module")
def prod():
    lib = _bind(rb.load())
    lib.fdtd_b200_subpixel_tensor3.argtypes = [D, PD, PD, PD, PD]
    lib.fdtd_b200_subpixel_tensor3.restype = C.c_int
    return lib


@pytest.fixture(scope="module")
def ref():
    if not oracle.ref_available():
        pytest.skip("rfsyn was not compiled here")
    return _bind(C.CDLL(str(oracle.REF_LIB)))


def _frac(lib, r, x, y, dx=1.0, dy=1.0):
    v = D(float("nan"))
    st = lib.subpixel_te_rectangle_fraction(C.byref(r), x, y, dx, dy, C.byref(v))
    return st, v.value


def _edge(lib, r, x, y, axis, length=1.0):
    v = D(float("nan"))
    st = lib.subpixel_te_rectangle_edge_fraction(C.byref(r), x, y, axis, length, C.byref(v))
    return st, v.value


def _tensor(lib, f, eb, ei, ang):
    a, b, c = D(), D(), D()
    st = lib.subpixel_te_mix_epsilon_tensor(f, eb, ei, ang, C.byref(a), C.byref(b), C.byref(c))
    return st, a.value, b.value, c.value


def test_rfsyn_subpixel_unit_test_against_the_product():
    exe = ROOT / "oracle" / "_ref" / "validators" / "subpixel_te_unit"
    if not exe.exists():
        pytest.skip("rfsyn's unit tests were not built here")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout == (ROOT / "tests" / "golden" / "validators" / "subpixel_te_unit.txt").read_text()


def test_edge_fraction_and_tensor_known_answers(prod):
    """The expectations of tests/subpixel_te_unit.c:572-631."""
    assert _edge(prod, Rect(0, 0, 2, 2, 0), -0.5, 0, 1) == (0, pytest.approx(1.0, abs=1e-14))
    assert _edge(prod, Rect(0, 0, 2, 2, 0), 0, -0.5, 2) == (0, pytest.approx(1.0, abs=1e-14))
    assert _edge(prod, Rect(0, 0, 2, 2, 0), 1.5, 0, 1) == (0, 0.0)
    # rfsyn's block expects 0.5 for the next two, but the edge [0, 1] x {0}
    # lies inside the rectangle [-1, 2] x [-0.5, 0.5] (rfsyn's own code also
    # returns 1), and the edge {0} x [0, 1] inside [-1.5, 1.5] x [0, 1]
    assert _edge(prod, Rect(0.5, 0, 3, 1, 0), 0, 0, 1) == (0, pytest.approx(1.0, abs=1e-14))
    assert _edge(prod, Rect(0, 0.5, 1, 3, math.pi / 2), 0, 0, 2) == (0, pytest.approx(1.0, abs=1e-14))
    e = D()
    assert prod.subpixel_te_mix_epsilon_harmonic(0.0, 1, 4, C.byref(e)) == 0 and e.value == 1.0
    assert prod.subpixel_te_mix_epsilon_harmonic(1.0, 1, 4, C.byref(e)) == 0 and e.value == 4.0
    assert prod.subpixel_te_mix_epsilon_harmonic(0.5, 1, 4, C.byref(e)) == 0 and abs(e.value - 1.6) <= 1e-14
    assert prod.subpixel_te_mix_epsilon_harmonic(1.1, 1, 4, C.byref(e)) == -1
    for q in range(2):
        st, xx, xy, yy = _tensor(prod, 0.0, 1, 4, q * 0.77)
        assert st == 0 and abs(xx - 1) <= 1e-14 and abs(yy - 1) <= 1e-14 and xy == 0.0
        st, xx, xy, yy = _tensor(prod, 1.0, 1, 4, q * 0.77)
        assert st == 0 and abs(xx - 0.25) <= 1e-14 and abs(yy - 0.25) <= 1e-14 and xy == 0.0
    st, xx, xy, yy = _tensor(prod, 0.5, 1, 4, 0.0)
    assert st == 0 and abs(xx - 0.625) <= 1e-14 and abs(yy - 0.4) <= 1e-14 and xy == 0.0
    st, xx, xy, yy = _tensor(prod, 0.5, 1, 4, math.pi / 2)
    assert st == 0 and abs(xx - 0.4) <= 1e-13 and abs(yy - 0.625) <= 1e-13 and abs(xy) <= 1e-13
    for q in range(1, 6):
        st, xx, xy, yy = _tensor(prod, 0.5, 1, 4, q * 0.31)
        assert st == 0 and abs(xx + yy - 1.025) <= 1e-13


def test_helpers_agree_with_rfsyn_on_random_inputs(prod, ref):
    rng = np.random.default_rng(7)
    for _ in range(4000):
        r = Rect(*rng.uniform(-2, 2, 2), *rng.uniform(0.05, 4, 2), rng.uniform(-4, 4))
        x, y = rng.uniform(-3, 3, 2)
        dx, dy = rng.uniform(0.2, 2, 2)
        sa, fa = _frac(prod, r, x, y, dx, dy)
        sb, fb = _frac(ref, r, x, y, dx, dy)
        assert sa == sb and abs(fa - fb) <= 1e-13, (fa, fb)
        length = rng.uniform(0.1, 2)
        r0 = Rect(r.center_x, r.center_y, r.size_u, r.size_v, 0.0)
        for axis in (1, 2):
            sa, ea = _edge(prod, r0, x, y, axis, length)
            sb, eb = _edge(ref, r0, x, y, axis, length)
            assert sa == sb and abs(ea - eb) <= 1e-13
        f, e1, e2, ang = rng.uniform(), rng.uniform(1, 12), rng.uniform(1, 12), rng.uniform(-4, 4)
        ta, tb = _tensor(prod, f, e1, e2, ang), _tensor(ref, f, e1, e2, ang)
        assert ta[0] == tb[0] and np.allclose(ta[1:], tb[1:], rtol=0, atol=1e-15)
        for fn in ("subpixel_te_mix_epsilon", "subpixel_te_mix_epsilon_harmonic"):
            va, vb = D(), D()
            assert getattr(prod, fn)(f, e1, e2, C.byref(va)) == getattr(ref, fn)(f, e1, e2, C.byref(vb)) == 0
            assert va.value == vb.value


def test_edge_fraction_is_the_geometric_share(prod):
    rng = np.random.default_rng(8)
    t = (np.arange(20000) + 0.5) / 20000
    for _ in range(300):
        r = Rect(*rng.uniform(-1, 1, 2), *rng.uniform(0.2, 3, 2), rng.uniform(-4, 4))
        x, y, length = *rng.uniform(-2, 2, 2), rng.uniform(0.2, 2)
        c, s_ = math.cos(r.angle_rad), math.sin(r.angle_rad)
        for axis in (1, 2):
            px = x + (t * length if axis == 1 else 0.0) - r.center_x
            py = y + (t * length if axis == 2 else 0.0) - r.center_y
            u, v = px * c + py * s_, py * c - px * s_
            want = np.mean((np.abs(u) <= r.size_u / 2) & (np.abs(v) <= r.size_v / 2))
            st, got = _edge(prod, r, x, y, axis, length)
            assert st == 0 and abs(got - want) <= 2e-4, (axis, got, want)


def test_error_codes_and_untouched_outputs(prod):
    v = D(0.123)
    assert prod.subpixel_te_rectangle_fraction(None, 0, 0, 1, 1, C.byref(v)) == -1
    assert prod.subpixel_te_rectangle_fraction(C.byref(Rect(0, 0, -1, 1, 0)), 0, 0, 1, 1, C.byref(v)) == -1
    assert prod.subpixel_te_rectangle_fraction(C.byref(Rect(-1.7e308, 0, 1, 1, 0)), 1.7e308, 0, 1, 1,
                                               C.byref(v)) == -2
    assert v.value == 0.123
    assert prod.subpixel_te_rectangle_edge_fraction(C.byref(Rect(0, 0, 1, 1, 0)), 0, 0, 3, 1.0, C.byref(v)) == -1
    e = D(9.0)
    assert prod.subpixel_te_mix_epsilon(0.5, 0.5, 4, C.byref(e)) == -1
    assert prod.subpixel_te_rectangle_epsilon(C.byref(Rect(0, 0, 1, 1, 0)), 0, 0, 1, 1, 1, 4, C.byref(v),
                                              C.byref(v)) == -1
    assert v.value == 0.123 and e.value == 9.0


def _t3(lib, f, eb, ei, n):
    arr = lambda a: (D * len(a))(*a)
    out = (D * 9)()
    st = lib.fdtd_b200_subpixel_tensor3(f, arr(np.ravel(eb)), arr(np.ravel(ei)), arr(n), out)
    return st, np.array(out[:]).reshape(3, 3)


def test_tensor3_z_invariant_limit_is_rfsyns_2x2_rule(prod, ref):
    rng = np.random.default_rng(11)
    for _ in range(500):
        f, e1, e2, ang = rng.uniform(), rng.uniform(1, 12), rng.uniform(1, 12), rng.uniform(-4, 4)
        st, m = _t3(prod, f, e1 * np.eye(3), e2 * np.eye(3), [math.cos(ang), math.sin(ang), 0.0])
        assert st == 0
        _, xx, xy, yy = _tensor(ref, f, e1, e2, ang)
        assert np.allclose([m[0, 0], m[0, 1], m[1, 0], m[1, 1]], [xx, xy, xy, yy], rtol=0, atol=1e-14)
        assert abs(m[2, 2] - 1.0 / ((1 - f) * e1 + f * e2)) <= 1e-14
        assert abs(m[0, 2]) <= 1e-15 and abs(m[1, 2]) <= 1e-15


def test_tensor3_isotropic_closed_form_and_ends(prod):
    rng = np.random.default_rng(12)
    for _ in range(500):
        f, e1, e2, n = rng.uniform(), rng.uniform(1, 12), rng.uniform(1, 12), rng.normal(size=3)
        st, m = _t3(prod, f, e1 * np.eye(3), e2 * np.eye(3), n)
        assert st == 0 and np.allclose(m, isotropic_minv(f, e1, e2, n), rtol=0, atol=1e-14)
    assert np.allclose(_t3(prod, 0.5, np.eye(3), 4 * np.eye(3), [1, 0, 0])[1], np.diag([0.625, 0.4, 0.4]))
    assert np.allclose(_t3(prod, 0.0, 2 * np.eye(3), 4 * np.eye(3), [0, 1, 1])[1], np.eye(3) / 2)
    assert np.allclose(_t3(prod, 1.0, 2 * np.eye(3), 4 * np.eye(3), [0, 1, 1])[1], np.eye(3) / 4)


def _spd(rng):
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    return q @ np.diag(rng.uniform(1.5, 10, 3)) @ q.T


def test_tensor3_anisotropic_equals_the_oracle_restatement(prod):
    rng = np.random.default_rng(13)
    for _ in range(500):
        eb = _spd(rng) if rng.uniform() < 0.5 else rng.uniform(1, 4) * np.eye(3)
        ei = _spd(rng)
        eb, ei = 0.5 * (eb + eb.T), 0.5 * (ei + ei.T)
        f, n = rng.uniform(), rng.normal(size=3)
        st, m = _t3(prod, f, eb, ei, n)
        assert st == 0
        want = smoothed_minv(f, eb, ei, n)
        assert np.allclose(m, want, rtol=1e-12, atol=1e-14), np.abs(m - want).max()
        assert np.allclose(m, m.T, atol=1e-15) and np.all(np.linalg.eigvalsh(m) > 0)


def test_tensor3_rejects_bad_arguments(prod):
    assert _t3(prod, 1.5, np.eye(3), np.eye(3), [1, 0, 0])[0] == -1
    assert _t3(prod, 0.5, np.eye(3), np.eye(3), [0, 0, 0])[0] == -1
    bad = np.eye(3)
    bad[0, 1] = 0.5  # not symmetric
    assert _t3(prod, 0.5, bad, np.eye(3), [1, 0, 0])[0] == -1
    assert _t3(prod, 0.5, -np.eye(3), np.eye(3), [1, 0, 0])[0] == -1
