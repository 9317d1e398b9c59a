"""Full 3x3 anisotropic permittivity (no rfsyn counterpart; rfsyn's tensor
edges are 2x2, materials.c:658-903).

CPU (oracle only), the physics that pins the restatement:
  * in the scope of rfsyn's 2x2 tensor edges (z-invariant TM field, uniform
    medium filling a periodic domain) the 3x3 update equals rfsyn's to
    rounding;
  * a diagonal 3x3 sample is the scalar medium (relative 1e-10 over the run);
  * a plane wave in a uniform rotated uniaxial medium keeps the polarisation
    of its eigenvector and travels at c / sqrt(eps) of that eigenvalue;
  * a closed cavity filled with a random symmetric positive-definite tensor
    stays bounded over thousands of steps.
CPU (product host side): the box helper's inverse of eps_r.
GPU: FP64 device runs equal the oracle bit for bit on scenes with rotated
anisotropic blocks (CPML, periodic axes, sources inside the block); FP32
within the FP32 bound."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle import Scene
from tests.cases import DT1, run_device


def rot(axis, ang):
    c, s = math.cos(ang), math.sin(ang)
    if axis == "z":
        return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1.0]])
    if axis == "x":
        return np.array([[1.0, 0, 0], [0, c, -s], [0, s, c]])
    return np.array([[c, 0, s], [0, 1.0, 0], [-s, 0, c]])


def inv_rows(eps):
    return np.linalg.inv(eps)


def block_rows(m, i0, i1, j0, j1, k0, k1):
    return [(c, i, j, k, tuple(m[c])) for i in range(i0, i1) for j in range(j0, j1) for k in range(k0, k1)
            for c in range(3)]


def _gd(t0, tau):
    return (0, t0 * DT1, tau * DT1, 0.0)


def aniso_scene(periodic=0, npml=3):
    R = rot("z", 0.4) @ rot("x", -0.7) @ rot("y", 0.3)
    eps = R @ np.diag([2.0, 5.0, 9.0]) @ R.T
    m = inv_rows(eps)
    s = Scene(nx=16, ny=14, nz=15, n_steps=70, npml=npml, periodic=periodic,
              sources=[(8, 7, 7, 2, 0, 1.0, *_gd(18, 5)), (8, 6, 8, 0, 0, 0.7, *_gd(25, 6))],
              probes=[(9, 7, 7, 2), (8, 8, 8, 0), (7, 7, 9, 1), (11, 7, 7, 4)], freqs=[20e9, 40e9])
    s.tensor3 = block_rows(m, 6, 11, 5, 10, 5, 11)
    return s


# ---------------------------------------------------------------- CPU --------
def test_diagonal_tensor_is_the_scalar_medium():
    base = dict(nx=12, ny=11, nz=10, n_steps=80, npml=2,
                sources=[(6, 5, 5, 2, 0, 1.0, *_gd(15, 4))], probes=[(7, 5, 5, 2), (6, 6, 4, 0)])
    a = Scene(boxes=[(4, 9, 3, 8, 3, 8, 4.0, 0.0)], **base)
    b = Scene(**base)
    b.tensor3 = block_rows(np.diag([0.25, 0.25, 0.25]), 4, 9, 3, 8, 3, 8)
    ta, tb = oracle.run_oracle(a)["td"], oracle.run_oracle(b)["td"]
    assert np.abs(ta - tb).max() <= 1e-10 * np.abs(ta).max()


def test_plane_wave_in_rotated_uniaxial_medium():
    """Periodic x / y, a sheet source of the eigen-polarisation e1 =
    (cos p, sin p, 0) of eps = Rz(p) diag(2.5, 6, 4) Rz(p)^T in a uniform
    medium: the far probe sees Ey / Ex = tan p (no conversion into the other
    eigenmode) and the pulse at the speed of sqrt(2.5)."""
    p, e1 = 0.5, 2.5
    R = rot("z", p)
    m = inv_rows(R @ np.diag([e1, 6.0, 4.0]) @ R.T)
    nz, z0, z1 = 420, 100, 300
    srcs = []
    for i in range(4):
        for j in range(4):
            srcs.append((i, j, z0, 0, 0, math.cos(p), *_gd(60, 15)))
            srcs.append((i, j, z0, 1, 0, math.sin(p), *_gd(60, 15)))
    s = Scene(nx=4, ny=4, nz=nz, n_steps=1100, periodic=3, sources=srcs,
              probes=[(1, 1, z0 + 20, 0), (1, 1, z0 + 20, 1), (1, 1, z1, 0), (1, 1, z1, 1)])
    s.tensor3 = block_rows(m, 0, 4, 0, 4, 1, nz - 1)
    td = oracle.run_oracle(s)["td"]
    ex, ey = td[2], td[3]
    assert np.abs(ex).max() > 0
    n = np.argmax(np.hypot(ex, ey))
    assert abs(ey[n] / ex[n] - math.tan(p)) < 1e-3 * math.tan(p)
    # cross-polarised part stays small over the whole record
    cross = -math.sin(p) * ex + math.cos(p) * ey
    assert np.abs(cross).max() < 1e-3 * np.abs(np.hypot(ex, ey)).max()
    # arrival: peak-to-peak delay of the direct pulse between the two probe
    # planes (windows end before the first reflection from the PEC ends
    # reaches either probe: ~670 steps near, ~1160 far)
    def centroid(e):
        w = e * e
        return float((np.arange(e.size) * w).sum() / w.sum())

    near = np.hypot(td[0], td[1])[:400]
    far = np.hypot(ex, ey)[:900]
    delay = (centroid(far) - centroid(near)) * s.dt
    v = (z1 - z0 - 20) * s.dx / delay
    # 2 %: Yee dispersion at ~17 cells per wavelength in the medium slows the
    # pulse by well under 1 %
    assert abs(v - 299792458.0 / math.sqrt(e1)) < 0.02 * 299792458.0 / math.sqrt(e1)


def test_random_tensor_cavity_stays_bounded():
    rng = np.random.default_rng(4)
    Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    eps = Q @ np.diag(rng.uniform(2, 10, 3)) @ Q.T
    s = Scene(nx=10, ny=9, nz=8, n_steps=3000, sources=[(5, 4, 4, 2, 0, 1.0, *_gd(10, 3))],
              probes=[(5, 4, 4, 2), (3, 3, 3, 0), (6, 5, 2, 1)])
    s.tensor3 = block_rows(inv_rows(eps), 1, 9, 1, 8, 1, 7)
    td = oracle.run_oracle(s)["td"]
    assert np.all(np.isfinite(td))
    early = np.abs(td[:, 300:1000]).max()
    late = np.abs(td[:, 2000:]).max()
    assert late < 2.0 * early


def test_reduces_to_rfsyn_2x2_tensor_in_its_scope():
    """rfsyn's tensor edges (materials.c:847-903) are the 2x2 (Ex, Ey)
    inverse permittivity of a z-invariant TM field, coupled to the four
    surrounding samples with the pair weight 0.25 rho sqrt(m11 m11'); in a
    uniform medium that fills a fully periodic domain the weight is 0.25 m12
    and the 3x3 rows (m11, m12, 0), (m12, m22, 0), (0, 0, 1/eps_z) describe
    the same update.  Driven z-invariantly (an Ex / Ey sheet along z), the two
    agree to rounding (1e-10 of the peak) at every probe."""
    eps = np.array([[4.0, 1.2], [1.2, 2.5]])
    m = np.linalg.inv(eps)
    eps_z = 3.0
    n, nz = 12, 3
    base = dict(nx=n, ny=n, nz=nz, n_steps=240, periodic=7,
                sources=[(5, 6, k, c, 0, 1.0 if c == 0 else 0.6, *_gd(25, 6)) for k in range(nz) for c in (0, 1)],
                probes=[(8, 4, 1, 0), (2, 9, 1, 1), (6, 6, 2, 5), (10, 10, 0, 0)])
    cells = [(i, j, k) for i in range(n) for j in range(n) for k in range(nz)]
    a = Scene(boxes=[(0, n, 0, n, 0, nz, eps_z, 0.0)],
              tensors=[(0, i, j, k, m[0, 0], m[0, 1], m[1, 1]) for (i, j, k) in cells] +
                      [(1, i, j, k, m[1, 1], m[0, 1], m[0, 0]) for (i, j, k) in cells], **base)
    b = Scene(**base)
    b.tensor3 = ([(0, i, j, k, (m[0, 0], m[0, 1], 0.0)) for (i, j, k) in cells] +
                 [(1, i, j, k, (m[0, 1], m[1, 1], 0.0)) for (i, j, k) in cells] +
                 [(2, i, j, k, (0.0, 0.0, 1.0 / eps_z)) for (i, j, k) in cells])
    ta, tb = oracle.run_oracle(a)["td"], oracle.run_oracle(b)["td"]
    peak = np.abs(ta).max()
    assert peak > 0
    assert np.abs(ta - tb).max() <= 1e-10 * peak, np.abs(ta - tb).max() / peak


def test_box_helper_inverts_eps():
    lib = rb.load()
    lib.fdtd_grid_create.restype = C.c_void_p
    lib.fdtd_grid_create.argtypes = [C.c_size_t] * 3 + [C.c_double, C.c_double]
    lib.materials_create.restype = C.c_void_p
    lib.materials_create.argtypes = [C.c_void_p]
    lib.fdtd_b200_materials_set_tensor3_box.argtypes = [C.c_void_p, C.c_void_p] + [C.c_size_t] * 6 + \
        [C.POINTER(C.c_double)]
    lib.fdtd_b200_materials_get_tensor3.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + [C.c_size_t] * 3 + \
        [C.POINTER(C.c_double)]
    g = lib.fdtd_grid_create(10, 10, 10, 1e-3, 0.99)
    m = lib.materials_create(g)
    R = rot("x", 0.3) @ rot("z", 1.1)
    eps = R @ np.diag([3.0, 7.0, 2.0]) @ R.T
    e = (C.c_double * 9)(*eps.ravel())
    assert lib.fdtd_b200_materials_set_tensor3_box(m, g, 2, 5, 2, 5, 2, 5, e) == 0
    row = (C.c_double * 3)()
    want = np.linalg.inv(eps)
    for c in range(3):
        assert lib.fdtd_b200_materials_get_tensor3(m, g, c, 3, 3, 3, row) == 0
        assert np.allclose(np.array(row[:]), want[c], rtol=1e-13, atol=1e-15)
    assert lib.fdtd_b200_materials_get_tensor3(m, g, 0, 7, 7, 7, row) == 1
    # not positive definite, and a cell on a face of an axis without wrap
    bad = (C.c_double * 9)(*np.diag([1.0, -2.0, 3.0]).ravel())
    assert lib.fdtd_b200_materials_set_tensor3_box(m, g, 2, 3, 2, 3, 2, 3, bad) == -1
    assert lib.fdtd_b200_materials_set_tensor3_box(m, g, 0, 2, 2, 3, 2, 3, e) == -1


# ---------------------------------------------------------------- GPU --------
@pytest.mark.gpu
@pytest.mark.parametrize("periodic", [0, 3, 4], ids=["cpml", "periodic_xy", "periodic_z"])
@pytest.mark.parametrize("schedule", [rb.FUSED, rb.SPLIT], ids=["fused", "split"])
def test_device_fp64_equals_oracle(periodic, schedule):
    s = aniso_scene(periodic=periodic, npml=0 if periodic else 3)
    want = oracle.run_oracle(s)
    got = run_device(s, rb.FP64, schedule)
    assert np.array_equal(got["td"], want["td"])


@pytest.mark.gpu
def test_device_fp32_within_bound():
    s = aniso_scene()
    want = oracle.run_oracle(s)["td"]
    got = run_device(s, rb.FP32, rb.FUSED)["td"]
    for p in range(want.shape[0]):
        scale = max(np.abs(want[p]).max(), 1e-30)
        assert np.abs(got[p] - want[p]).max() / scale < 1e-3
