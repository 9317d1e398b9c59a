"""FP32 accuracy at the sizes the benchmark runs.

The full C2 scene (256^3, 27 spheres, 4000 steps, 16 probes x 256 DFT bins)
and the full C3 periodic cell (128 x 128 x 512, TF/SF plane wave, tilted 3x3
slab, Lorentz layer, 6000 steps, 2 x 64 probes x 512 bins) are run twice on
the GPU: in FP32 (the benchmarked precision) and in FP64.  The FP64 device
loop equals rfsyn's double-precision loop and the CPU oracle bit for bit at
every size they can run (tests/test_gpu_parity.py, tests/test_c2_scaled.py,
tests/test_c3_scaled.py), so at these sizes it stands in for the oracle.
Bound: every probe's spectrum within 1e-4 relative L2 of its FP64 spectrum,
each probe normalised by its own FP64 norm."""
from __future__ import annotations

import numpy as np
import pytest

import rfsyn_b200 as rb
from rfsyn_b200 import scenes

pytestmark = pytest.mark.gpu
FP32_SPEC_L2 = 1e-4


def _spectra(w):
    st = scenes.scene_setup(w)
    r = rb.run(scenes.run_config(w), st.ptr if st else None, None)
    return r["dft"], r["td"]


def _rel_l2(got, want):
    return np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)


@pytest.mark.parametrize("recipe", ["c2", "c3"])
def test_full_size_fp32_spectra_against_fp64(recipe):
    make = getattr(scenes, recipe)
    s32, td32 = _spectra(make(precision=rb.FP32))
    s64, td64 = _spectra(make(precision=rb.FP64))
    assert np.all(np.isfinite(td32)) and np.all(np.isfinite(td64))
    assert np.all(np.linalg.norm(s64, axis=1) > 0), "a probe saw no field"
    err = _rel_l2(s32, s64)
    print(f"{recipe}: FP32 spectrum relative L2 vs FP64, per probe: max {err.max():.3e}, "
          f"median {np.median(err):.3e}")
    assert err.max() <= FP32_SPEC_L2, (recipe, int(err.argmax()), float(err.max()))
