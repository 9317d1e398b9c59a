"""Host-side parts of the transfer-function surrogate (no GPU): the source
spectrum the transfer functions are divided by, and the scene vector."""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from rfsyn_b200 import surrogate as sg


def _direct_spectrum(w) -> np.ndarray:
    s = w.sources[0]
    t = np.arange(w.n_steps) * w.dt
    u = (t - s["p1"]) / s["p2"]
    v = s["amplitude"] * np.exp(-u * u) * np.sin(2.0 * math.pi * s["p0"] * (t - s["p1"]))
    f = np.asarray(w.freqs)
    return (v[None, :] * np.exp(-2j * math.pi * f[:, None] * t[None, :])).sum(axis=1) * w.dt


def test_source_spectrum_is_the_waveform_transform_shared_between_scenes():
    ws = sg.c5_scenes(seed=52, n_scenes=6)
    specs = [sg.source_spectrum(w) for w in ws]
    assert np.array_equal(specs[3], _direct_spectrum(ws[3]))
    # every surrogate scene has the same waveform, dt, steps and bins: one array
    assert all(s is specs[0] for s in specs)
    assert not specs[0].flags.writeable
    # another waveform gets its own spectrum
    w = ws[0]
    src = dict(w.sources[0], p0=5e9)
    other = dataclasses.replace(w, sources=[src])
    so = sg.source_spectrum(other)
    assert so is not specs[0]
    assert np.array_equal(so, _direct_spectrum(other))


def test_scene_vector_ignores_the_order_scatterers_are_listed_in():
    ws = sg.c5_scenes(seed=7, n_scenes=40)
    w = next(x for x in ws if len(x.spheres) >= 3)
    flipped = dataclasses.replace(w, spheres=list(reversed(w.spheres)))
    for rx in range(len(w.probes)):
        a, b = sg.features(w, rx), sg.features(flipped, rx)
        assert a.shape == (sg.N_FEAT,)
        assert np.array_equal(a, b)
        # rows sorted by excess path length, padding rows zero
        ex = a[2:6 * len(w.spheres):6]
        assert np.all(np.diff(ex) >= 0)
        assert not a[6 * len(w.spheres):48].any()
