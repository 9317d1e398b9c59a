"""The library's device memory cache: blocks that a destroyed simulation
freed (1 MB and more rounded to 2 MB, smaller ones to a power of two) are
handed to the next creation, still holding
the previous simulation's fields, PML state and scene arrays.  A simulation
built on reused blocks must give the same probe series and spectra, bit for
bit, as the same simulation built on fresh memory, and releasing the cache
returns every block to the driver."""
from __future__ import annotations

import numpy as np
import pytest

import rfsyn_b200 as rb
from rfsyn_b200 import scenes

pytestmark = pytest.mark.gpu


def _run(w):
    setup = scenes.scene_setup(w)
    sim = rb.Sim(scenes.run_config(w), setup.ptr if setup else None, None)
    try:
        sim.advance(w.n_steps)
        return sim.probes(), sim.dft()
    finally:
        sim.close()


@pytest.mark.parametrize("precision", [rb.FP32, rb.FP64], ids=["fp32", "fp64"])
def test_reused_blocks_give_identical_results(precision):
    a, b = scenes.c4(seed=21, n_scenes=2, precision=precision, n_steps=160, lo=60, hi=64, npml=8)
    rb.release_cached_memory()
    assert rb.cached_bytes() == 0
    td0, dft0 = _run(a)                  # fresh blocks from the driver
    assert rb.cached_bytes() >= 12 << 20  # the field block at least is kept
    _run(b)                              # another scene dirties the cached blocks
    td1, dft1 = _run(a)                  # the first scene again, on reused blocks
    assert np.isfinite(td0).all() and np.abs(td0).max() > 0
    assert np.array_equal(td0, td1)
    assert np.array_equal(dft0, dft1)
    rb.release_cached_memory()
    assert rb.cached_bytes() == 0
