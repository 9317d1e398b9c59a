"""Heightmap worlds mapped onto the FDTD materials
(fdtd_b200_materials_apply_heightmap; rfsyn has the world, engine/world/
world.c, but never applies it to a grid).

CPU:
  * a numpy restatement of world.c's cell description (solid fraction, bulk
    id, surface normal) equals rfsyn's own world_get_cell, compiled from its
    sources into oracle/_ref, on random heightmaps; it also reproduces the
    expectations of rfsyn's tests/world_unit.c;
  * the product's per-component coefficients equal the restatement's (bulk
    ids, and the diagonal smoothing of cut cells) exactly;
  * the product rejects what world_create_heightmap rejects.
GPU: an FP64 run of a terrain scene equals the CPU oracle given the same
materials as boxes and per-component overrides, bit for bit."""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
import rfsyn_b200 as rb
from oracle import Scene
from tests.cases import DT1, scene_run_config

EPS0 = 8.8541878128e-12
REF_LIB = Path(oracle.__file__).resolve().parent / "_ref" / "librfsyn_ref.so"


# ---------------------------------------------------------------- restatement
def world_cells(heights: np.ndarray, columns: np.ndarray, nz: int, dx: float, air: int = 0):
    """Per cell (i, j, k): solid fraction f, bulk id, and for 0 < f < 1 the
    surface normal (world.c:23-47, :92-110)."""
    nx, ny = heights.shape
    hc = np.minimum(heights / dx, float(nz))
    f = np.clip(hc[:, :, None] - np.arange(nz)[None, None, :], 0.0, 1.0)
    bulk = np.where(f >= 0.5, columns[:, :, None], air)
    il = np.maximum(np.arange(nx) - 1, 0)
    ir = np.minimum(np.arange(nx) + 1, nx - 1)
    jl = np.maximum(np.arange(ny) - 1, 0)
    jr = np.minimum(np.arange(ny) + 1, ny - 1)
    gx = np.where((ir != il)[:, None], (heights[ir, :] - heights[il, :]) / ((ir - il)[:, None] * dx), 0.0)
    gy = np.where((jr != jl)[None, :], (heights[:, jr] - heights[:, jl]) / ((jr - jl)[None, :] * dx), 0.0)
    length = np.hypot(np.hypot(gx, gy), 1.0)
    normal = np.stack([-gx / length, -gy / length, 1.0 / length], axis=-1)
    return f, bulk, normal


def expected_media(heights, columns, media, nz, dx, air=0, smoothing=1):
    """(eps_r, sigma) of every component c of every cell: [nx, ny, nz, 3, 2],
    the product's rule (bulk id; cut cells: diagonal of the smoothed inverse
    permittivity, arithmetic sigma)."""
    f, bulk, normal = world_cells(heights, columns, nz, dx, air)
    nx, ny = heights.shape
    out = np.zeros((nx, ny, nz, 3, 2))
    for i in range(nx):
        for j in range(ny):
            es, ss = media[columns[i, j]]
            ea, sa = media[air]
            for k in range(nz):
                fk = float(f[i, j, k])
                for c in range(3):
                    if smoothing and 0.0 < fk < 1.0:
                        n2 = float(normal[i, j, c]) * float(normal[i, j, c])
                        mean = fk * es + (1.0 - fk) * ea
                        minv = fk / es + (1.0 - fk) / ea
                        inv = n2 * minv + (1.0 - n2) / mean
                        out[i, j, k, c] = (1.0 / inv, fk * ss + (1.0 - fk) * sa)
                    else:
                        out[i, j, k, c] = media[int(bulk[i, j, k])]
    return out


def make_coeff(eps_r, sigma, dt, dx):
    """rfsyn materials.c:92-125."""
    eps = eps_r * EPS0
    loss = (sigma * dt) / (2.0 * eps)
    cb = dt / (eps * dx)
    return (1.0 - loss) / (1.0 + loss), cb / (1.0 + loss)


def terrain(nx, ny, nz, seed, lo=2.0, hi=None, n_ids=3):
    rng = np.random.default_rng(seed)
    hi = nz - 2.0 if hi is None else hi
    x = np.arange(nx)[:, None]
    y = np.arange(ny)[None, :]
    cells = lo + (hi - lo) * (0.5 + 0.3 * np.sin(0.7 * x + 0.2) * np.cos(0.5 * y) + 0.15 * rng.random((nx, ny)))
    columns = rng.integers(1, n_ids + 1, size=(nx, ny)).astype(np.uint8)
    return cells, columns


# ---------------------------------------------------------------- CPU --------
class _WorldCell(C.Structure):
    _fields_ = [("ids", C.c_uint8 * 2), ("fractions", C.c_double * 2), ("count", C.c_size_t),
                ("normal", C.c_double * 3)]


class _WorldCfg(C.Structure):
    _fields_ = [("nx", C.c_size_t), ("ny", C.c_size_t), ("nz", C.c_size_t), ("dx", C.c_double),
                ("heights_m", C.POINTER(C.c_double)), ("column_materials", C.POINTER(C.c_uint8)),
                ("air_id", C.c_uint8)]


@pytest.mark.skipif(not REF_LIB.exists(), reason="rfsyn not compiled into oracle/_ref")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restatement_equals_rfsyn_world(seed):
    ref = C.CDLL(str(REF_LIB))
    ref.world_create_heightmap.restype = C.c_void_p
    ref.world_create_heightmap.argtypes = [C.POINTER(_WorldCfg)]
    ref.world_get_cell.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.POINTER(_WorldCell)]
    ref.world_destroy.argtypes = [C.c_void_p]
    ref.world_mixed_cell_count.restype = C.c_size_t
    ref.world_mixed_cell_count.argtypes = [C.c_void_p]
    nx, ny, nz, dx = 7, 5, 9, 2e-3
    cells, columns = terrain(nx, ny, nz, seed)
    cells[0, 0] = 0.0
    columns[0, 0] = 0                      # an air column
    cells[2, 3] = 4.0                      # a flat top on a cell face
    heights = np.ascontiguousarray(cells * dx)
    cfg = _WorldCfg(nx, ny, nz, dx, heights.ctypes.data_as(C.POINTER(C.c_double)),
                    columns.ctypes.data_as(C.POINTER(C.c_uint8)), 0)
    w = ref.world_create_heightmap(C.byref(cfg))
    assert w
    try:
        f, bulk, normal = world_cells(heights, columns, nz, dx)
        mixed = 0
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    cell = _WorldCell()
                    assert ref.world_get_cell(w, i, j, k, C.byref(cell)) == 0
                    if cell.count == 2:
                        mixed += 1
                        assert cell.fractions[0] == f[i, j, k]
                        assert cell.ids[0] == columns[i, j]
                        assert list(cell.normal) == list(normal[i, j])
                    else:
                        assert f[i, j, k] in (0.0, 1.0)
                        assert cell.ids[0] == bulk[i, j, k]
        assert mixed == ref.world_mixed_cell_count(w)
    finally:
        ref.world_destroy(w)


def test_restatement_reproduces_rfsyn_world_unit():
    # tests/world_unit.c: flat 1.25 m on a 3 x 2 x 4 world at dx 1 m
    h = np.full((3, 2), 1.25)
    ids = np.ones((3, 2), dtype=np.uint8)
    f, bulk, normal = world_cells(h, ids, 4, 1.0)
    assert abs(f.sum() * 1.0 - 7.5) < 1e-12
    assert int(((f > 0) & (f < 1)).sum()) == 6
    assert bulk[0, 0, 0] == 1 and bulk[0, 0, 1] == 0 and f[0, 0, 1] == 0.25
    assert np.allclose(normal[0, 0], [0.0, 0.0, 1.0])
    # linear ramp 0.25 + i: normal (-1, 0, 1) / sqrt 2 at the middle column
    h = np.array([[0.25 + i] * 2 for i in range(3)])
    ids[1, 0] = 2
    f, bulk, normal = world_cells(h, ids, 4, 1.0)
    assert abs(f.sum() - 7.5) < 1e-12
    assert abs(normal[1, 0, 0] + 1 / math.sqrt(2)) < 1e-12 and abs(normal[1, 0, 2] - 1 / math.sqrt(2)) < 1e-12


def _grid_and_materials(nx, ny, nz, dx):
    lib = rb.load()
    lib.fdtd_grid_create.restype = C.c_void_p
    lib.fdtd_grid_create.argtypes = [C.c_size_t] * 3 + [C.c_double, C.c_double]
    lib.materials_create.restype = C.c_void_p
    lib.materials_create.argtypes = [C.c_void_p]
    lib.materials_get_coefficients.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + [C.c_size_t] * 3 + \
        [C.POINTER(C.c_double * 2)]
    lib.fdtd_grid_destroy.argtypes = [C.c_void_p]
    lib.materials_destroy.argtypes = [C.c_void_p]
    g = lib.fdtd_grid_create(nx, ny, nz, dx, 0.99)
    return lib, g, lib.materials_create(g)


def _apply(lib, g, m, cells, columns, media, nz, dx, smoothing=1, air=0, hdx=None):
    h = np.ascontiguousarray(cells * dx)
    ids = np.ascontiguousarray(columns, dtype=np.uint8)
    hm = rb.Heightmap(h.shape[0], h.shape[1], nz, dx if hdx is None else hdx, h.ctypes.data_as(C.POINTER(C.c_double)),
                      ids.ctypes.data_as(C.POINTER(C.c_uint8)), air)
    med = (rb.Medium * len(media))(*[rb.Medium(e, s) for e, s in media])
    mixed = C.c_size_t(0)
    rc = lib.fdtd_b200_materials_apply_heightmap(C.c_void_p(m), C.c_void_p(g), C.byref(hm), med, len(media),
                                                 smoothing, C.byref(mixed))
    return rc, mixed.value


MEDIA = [(1.0, 0.0), (4.28, 0.02665), (5.24, 0.0462), (30.29, 0.17151)]


@pytest.mark.parametrize("smoothing", [1, 0])
def test_product_coefficients_equal_restatement(smoothing):
    nx, ny, nz, dx = 9, 8, 10, 1e-3
    cells, columns = terrain(nx, ny, nz, 5)
    lib, g, m = _grid_and_materials(nx, ny, nz, dx)
    try:
        rc, mixed = _apply(lib, g, m, cells, columns, MEDIA, nz, dx, smoothing)
        assert rc == 0, rb.last_error()
        f, _, _ = world_cells(cells * dx, columns, nz, dx)
        assert mixed == int(((f > 0) & (f < 1)).sum()) > 0
        want = expected_media(cells * dx, columns, MEDIA, nz, dx, smoothing=smoothing)
        dt = 0.99 * (dx / (299792458.0 * math.sqrt(3.0)))
        out = (C.c_double * 2)()
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    for c in range(3):
                        if (c != 0 and i == 0) or (c != 1 and j == 0) or (c != 2 and k == 0):
                            continue          # PEC walls: samples rfsyn never updates
                        assert lib.materials_get_coefficients(C.c_void_p(m), C.c_void_p(g), c, i, j, k, out) == 0
                        ca, cb = make_coeff(*want[i, j, k, c], dt, dx)
                        assert (out[0], out[1]) == (ca, cb), (i, j, k, c)
    finally:
        lib.materials_destroy(m)
        lib.fdtd_grid_destroy(g)


def test_rejects_what_rfsyn_world_rejects():
    nx, ny, nz, dx = 4, 3, 5, 1e-3
    lib, g, m = _grid_and_materials(nx, ny, nz, dx)
    try:
        cells = np.full((nx, ny), 2.5)
        cols = np.ones((nx, ny), dtype=np.uint8)
        assert _apply(lib, g, m, cells, cols, MEDIA, nz, dx)[0] == 0
        for bad in (np.nan, -1.0, nz + 0.5):
            c2 = cells.copy()
            c2[1, 1] = bad
            assert _apply(lib, g, m, c2, cols, MEDIA, nz, dx)[0] == -1
        air_col = cols.copy()
        air_col[2, 0] = 0                  # air column with a height
        assert _apply(lib, g, m, cells, air_col, MEDIA, nz, dx)[0] == -1
        assert "height or material" in rb.last_error()
        missing = cols.copy()
        missing[0, 0] = 7                  # no medium for id 7
        assert _apply(lib, g, m, cells, missing, MEDIA, nz, dx)[0] == -1
        assert _apply(lib, g, m, cells, cols, MEDIA, nz, dx, hdx=2e-3)[0] == -1
        assert _apply(lib, g, m, cells, cols, [(0.5, 0.0), (4.0, 0.0)], nz, dx)[0] == -1   # eps_r < 1
    finally:
        lib.materials_destroy(m)
        lib.fdtd_grid_destroy(g)


# ---------------------------------------------------------------- GPU --------
def terrain_scene(nx=26, ny=22, nz=24, npml=4, n_steps=140):
    cells, columns = terrain(nx, ny, nz, 11, lo=6.0, hi=12.0)
    dx = 1e-3
    want = expected_media(cells * dx, columns, MEDIA, nz, dx)
    f, bulk, _ = world_cells(cells * dx, columns, nz, dx)
    boxes, comps = [], []
    for i in range(nx):
        for j in range(ny):
            kb = int((f[i, j] >= 0.5).sum())
            if kb:
                boxes.append((i, i + 1, j, j + 1, 0, kb, *MEDIA[columns[i, j]]))
            for k in range(nz):
                if 0.0 < f[i, j, k] < 1.0:
                    for c in range(3):
                        if (c != 0 and i == 0) or (c != 1 and j == 0) or (c != 2 and k == 0):
                            continue
                        comps.append((c, i, j, k, *want[i, j, k, c]))
    s = Scene(nx=nx, ny=ny, nz=nz, n_steps=n_steps, npml=npml, boxes=boxes, comps=comps,
              sources=[(13, 11, 18, 2, 0, 1.0, 0, 30 * DT1, 8 * DT1, 0.0)],
              probes=[(15, 11, 16, 2), (10, 9, 8, 0), (13, 14, 10, 1), (6, 6, 19, 2)], freqs=[20e9, 40e9])
    return s, cells, columns


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [rb.FUSED, rb.SPLIT], ids=["fused", "split"])
def test_device_fp64_terrain_equals_oracle(schedule):
    s, cells, columns = terrain_scene()
    want = oracle.run_oracle(s)
    setup = rb.HeightmapSetup(cells * 1e-3, columns, MEDIA, nz=s.nz, dx=1e-3)
    got = rb.run(scene_run_config(s, rb.FP64, schedule), setup.ptr)
    assert setup.mixed > 0
    assert np.array_equal(got["td"], want["td"])
    assert np.abs(want["td"]).max() > 0
