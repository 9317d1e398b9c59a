"""Multi-rank plumbing of the benches (rfsyn_b200.ranks) with two gloo ranks
on CPU: the path shards by scene, so the checks are that ranks get disjoint
shards and different scenes, and that the timing reduction and the
weak-scaling rate come out the same on every rank; for the surrogate's
pipeline, that uneven blocks gather in rank order, that the sharded data
generation reproduces the one-rank rows (the FDTD replaced by a stand-in)
and that the ensemble's members split over the ranks once.  Rendezvous on
127.0.0.1."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from rfsyn_b200 import ranks


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r = ranks.from_env()
    ranks.init(r, "gloo", timeout_s=60)
    try:
        import numpy as np

        from rfsyn_b200 import scenes

        # each rank builds its own scenes; the C2 recipe seeded per rank
        w = scenes.c2(seed=ranks.scene_seed(2, r))
        sig = float(np.sum([s[3] for s in w.spheres]))          # sum of radii identifies the scene
        ms_local = 10.0 + 5.0 * rank                              # the slower rank sets the time
        ms = ranks.max_over(r, ms_local, device="cpu")
        total = ranks.sum_over(r, float(rank + 1), device="cpu")
        rate = ranks.weak_rate(1000.0, ms, r)
        ranks.barrier(r)
        out.put((rank, list(ranks.shard(10, r)), sig, ms, total, rate))
    finally:
        ranks.finish(r)


def test_two_gloo_ranks_shard_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    shards = [x[1] for x in res]
    assert sorted(shards[0] + shards[1]) == list(range(10)) and not set(shards[0]) & set(shards[1])
    assert res[0][2] != res[1][2]                      # different scenes per rank
    for _, _, _, ms, total, rate in res:
        assert ms == 15.0 and total == 3.0            # max and sum over ranks, on every rank
        assert rate == pytest.approx(2 * 1000.0 / 0.015)


@pytest.mark.parametrize("n,world", [(10, 3), (7, 7), (3, 5), (0, 2)])
def test_shards_cover_once(n, world):
    got = []
    for r in range(world):
        got += list(ranks.shard(n, ranks.Ranks(r, world, r)))
    assert got == list(range(n))
    sizes = [len(ranks.shard(n, ranks.Ranks(r, world, r))) for r in range(world)]
    assert max(sizes) - min(sizes) <= 1


def test_single_rank_needs_no_process_group():
    r = ranks.Ranks(0, 1, 0)
    ranks.init(r)
    assert ranks.max_over(r, 3.5) == 3.5 and ranks.sum_over(r, 2.0) == 2.0
    ranks.barrier(r)
    ranks.finish(r)


def _fake_tf(ws, timings=None):
    """Stands in for the batched FDTD: rows determined by the scene's name
    (4 receivers each), so any sharding must reproduce them in order."""
    import numpy as np

    X, H = [], []
    for w in ws:
        s = int(w.name.replace("c5_scene", ""))
        for rx in range(4):
            X.append(np.full(54, s + 0.25 * rx))
            H.append(np.exp(1j * np.arange(256) * (s + 1)) * (rx + 1))
    return np.asarray(X), np.asarray(H)


def _pipeline_worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r = ranks.from_env()
    ranks.init(r, "gloo", timeout_s=60)
    try:
        import numpy as np

        from rfsyn_b200 import surrogate as sg

        # uneven blocks of several dtypes and shapes gather in rank order
        a = np.arange(3 + 2 * rank, dtype=np.float32) + 100 * rank
        c = (np.arange(6 * (1 + rank)).reshape(-1, 2, 3) + 1j * rank).astype(np.complex128)
        ga, gc = ranks.gather_rows(r, a, device="cpu"), ranks.gather_rows(r, c, device="cpu")
        want_a = np.concatenate([np.arange(3, dtype=np.float32), np.arange(5, dtype=np.float32) + 100])
        want_c = np.concatenate([np.arange(6).reshape(-1, 2, 3) + 0j, np.arange(12).reshape(-1, 2, 3) + 1j])
        # the surrogate's sharded data generation equals the one-rank run
        ws = sg.c5_scenes(seed=5, n_scenes=7)
        X, H = sg.sharded_transfer_functions(ws, r, device="cpu", tf=_fake_tf)
        X1, H1 = _fake_tf(ws)
        # results are compared here: only small values cross the queue
        out.put((rank, bool(np.array_equal(ga, want_a)), bool(np.array_equal(gc, want_c)),
                 bool(np.array_equal(X, X1)), bool(np.array_equal(H, H1)), ranks.members_of(5, r)))
    finally:
        ranks.finish(r)


def test_two_gloo_ranks_gather_the_surrogate_pipeline():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_pipeline_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    for rank, ok_a, ok_c, ok_x, ok_h, members in res:
        assert ok_a and ok_c and ok_x and ok_h, (rank, ok_a, ok_c, ok_x, ok_h)
    assert sorted(res[0][5] + res[1][5]) == list(range(5)) and not set(res[0][5]) & set(res[1][5])
