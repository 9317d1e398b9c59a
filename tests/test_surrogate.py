"""The transfer-function surrogate end to end on a small scene family
(transmitter / receiver positions varying in vacuum): training data from
the batched FDTD, a GPU-trained ensemble, and FDTD fallback wherever the
ensemble disagrees.  Checks that the ensemble learns the family (held-out
relative error), that the fallback returns exactly the FDTD transfer
functions, and what the network gains: its per-scene time against the
FDTD's."""
from __future__ import annotations

import numpy as np
import pytest

from rfsyn_b200 import surrogate as sg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    ws = sg.c5_scenes(seed=21, n_scenes=96, n=32, n_steps=600, npml=6, max_scat=0)
    timings = {}
    X, H = sg.transfer_functions(ws, timings=timings)
    G = sg.scene_transfer_targets(ws, H)
    ntr = 80 * 4
    sur = sg.Surrogate(members=3, width=128, depth=3, seed=1)
    losses = sur.fit(X[:ntr], G[:ntr], steps=3000, batch=64, lr=2e-3)
    yield dict(ws=ws, X=X, H=H, G=G, ntr=ntr, sur=sur, losses=losses, fdtd_ms=timings["fdtd_ms"])
    sur.close()


def test_ensemble_learns_the_family(trained):
    t = trained
    ws_te = t["ws"][80:]
    pred = t["sur"].predict(ws_te, t["X"][t["ntr"]:])
    err = sg.rel_err(pred.H, t["H"][t["ntr"]:])
    assert np.median(err) < 0.25, np.median(err)
    # disagreement tracks error: the rows the ensemble agrees on are the good ones
    lo = pred.spread <= np.median(pred.spread)
    assert err[lo].mean() <= err[~lo].mean() * 1.5


def test_fallback_returns_fdtd_where_unsure(trained):
    t = trained
    ws_te = t["ws"][80:88]
    pred = t["sur"].predict(ws_te)
    # a scene falls back when any of its receivers is unsure: threshold at
    # the median of the per-scene largest spread
    thr = float(np.median(pred.spread.reshape(len(ws_te), 4).max(axis=1)))
    res = sg.infer_with_fallback(t["sur"], ws_te, threshold=thr)
    rows = np.arange(len(ws_te) * 4).reshape(len(ws_te), 4)
    fell = set(res["fallback"])
    assert 0 < len(fell) < len(ws_te)
    H_ref = t["H"][t["ntr"]: t["ntr"] + 4 * len(ws_te)]
    for q in range(len(ws_te)):
        if q in fell:
            assert np.array_equal(res["H"][rows[q]], H_ref[rows[q]])
        else:
            assert np.allclose(res["H"][rows[q]], pred.H[rows[q]])
            assert np.all(pred.spread[rows[q]] <= thr)


def test_network_is_faster_than_fdtd(trained):
    """The gain of the surrogate: network inference per scene vs the batched
    FDTD per scene that produced the training data."""
    t = trained
    ws = t["ws"]
    import time

    t0 = time.perf_counter()
    t["sur"].predict(ws)
    sur_s = (time.perf_counter() - t0) / len(ws)
    fdtd_s = t["fdtd_ms"] / 1e3 / len(ws)
    assert sur_s < fdtd_s, (sur_s, fdtd_s)
