"""The CPU oracle against rfsyn's golden outputs (CPU only).

The golden fixtures were produced by rfsyn itself (tests/golden/
make_golden.py); where rfsyn's sources are present the oracle is also
compared with a live rfsyn build on fresh inputs.  The bar is bit-for-bit.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle
from tests.cases import CASES, c1_scene
from oracle import Scene

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(name):
    g = np.load(GOLDEN / f"{name}.npz")
    r = oracle.run_oracle(CASES[name])
    assert np.array_equal(r["td"], g["td"])
    assert np.array_equal(r["dft"], g["dft"])


def test_oracle_reproduces_simulate_unit_golden():
    # rfsyn's fdtd_simulate_echo: default CPML (kappa_max 7), Gaussian
    # derivative t0 = 40 dt, tau = 8 dt, t = n dt (simulate.c:37-38)
    dt = Scene(nx=1, ny=1, nz=1).dt
    s = Scene(nx=50, ny=50, nz=50, n_steps=200, npml=8, sources=[(25, 25, 25, 2, 0, 1.0, 0, 40 * dt, 8 * dt, 0)],
              probes=[(31, 25, 25, 2)])
    g = np.load(GOLDEN / "simulate_unit.npz")
    r = oracle.run_oracle(s)
    assert np.array_equal(r["td"][0], g["td"])


def test_oracle_reproduces_c1_golden():
    g = np.load(GOLDEN / "c1.npz")
    r = oracle.run_oracle(c1_scene())
    assert np.array_equal(r["td"], g["td"])
    assert np.array_equal(r["dft"], g["dft"])


def _pattern_fields(nx, ny, nz, seed=7):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1e-3, 1e-3, size=(6, nx + 1, ny + 1, nz + 1))


@pytest.mark.skipif(not oracle.ref_available(), reason="rfsyn sources not built here")
@pytest.mark.parametrize("mask", range(8))
def test_oracle_fields_match_rfsyn_all_periodic_masks(mask):
    # rfsyn tests/periodic_wrapping_unit.c: every periodic mask on a 5x6x7
    # grid, arbitrary initial fields, with CPML on the open axes
    s = Scene(nx=5, ny=6, nz=7, n_steps=3, periodic=mask, npml=1,
              boxes=[(1, 3, 1, 4, 2, 5, 3.0, 0.02)], comps=[(0, 2, 2, 2, 5.0, 0.0), (2, 1, 3, 3, 2.0, 0.1)])
    ini = _pattern_fields(5, 6, 7)
    a = oracle.fields_oracle(s, ini)
    b = oracle.fields_ref(s, ini)
    assert np.array_equal(a, b)


@pytest.mark.skipif(not oracle.ref_available(), reason="rfsyn sources not built here")
def test_oracle_matches_rfsyn_on_seeded_random_scenes():
    rng = np.random.default_rng(11)
    for trial in range(4):
        nx, ny, nz = (int(v) for v in rng.integers(9, 16, size=3))
        per = int(rng.integers(0, 8))
        boxes = []
        for _ in range(3):
            i0, j0, k0 = (int(rng.integers(0, n - 2)) for n in (nx, ny, nz))
            boxes.append((i0, i0 + 3, j0, j0 + 3, k0, k0 + 2, float(rng.uniform(1, 8)), float(rng.uniform(0, 0.05))))
        comps = [(int(rng.integers(0, 3)), int(rng.integers(1, nx - 1)), int(rng.integers(1, ny - 1)),
                  int(rng.integers(1, nz - 1)), float(rng.uniform(1, 10)), 0.0) for _ in range(5)]
        dt = Scene(nx=1, ny=1, nz=1).dt
        s = Scene(nx=nx, ny=ny, nz=nz, n_steps=40, periodic=per, npml=2, kappa_max=float(rng.uniform(1, 8)),
                  boxes=boxes, comps=comps,
                  sources=[(nx // 2, ny // 2, nz // 2, int(rng.integers(0, 3)), 0, 1.0, 0, 10 * dt, 3 * dt, 0)],
                  probes=[(1, 1, 1, 2), (nx // 2 + 1, ny // 2, nz // 2, int(rng.integers(0, 6)))],
                  freqs=[30e9, 60e9])
        a, b = oracle.run_oracle(s), oracle.run_ref(s)
        assert np.array_equal(a["td"], b["td"]), trial
        assert np.array_equal(a["dft"], b["dft"]), trial
