"""One process per GPU over scenes: the multi-GPU plumbing of the benches.

The FDTD path shards by scene -- every scene is an independent unit with no
exchange between ranks -- so around the time loop the only collectives are
a barrier around the timed region and the max over ranks of the elapsed
time (a weak-scaling throughput is every rank's units over the slowest
rank's time).  The surrogate's pipeline shards its scene set the same way
and then exchanges data: the training rows every rank generated are
gathered on every rank (gather_rows), the ensemble's members are split over
the ranks (members_of) and their predictions gathered.  The backend is NCCL
on GPUs; the same functions run over gloo on CPU, which is how the
multi-rank logic is tested without several GPUs.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local: int


def from_env() -> Ranks:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (1 process if unset)."""
    return Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def init(r: Ranks, backend: str = "nccl", timeout_s: int = 120) -> None:
    """Joins the process group when there is more than one rank.  A short
    timeout makes a rank that never arrives end the others' next collective
    with an error instead of a hang."""
    if r.world > 1:
        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over(r: Ranks, x: float, device: str = "cuda") -> float:
    """The maximum of x over all ranks (x itself with one rank)."""
    if r.world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over(r: Ranks, x: float, device: str = "cuda") -> float:
    """The sum of x over all ranks (x itself with one rank)."""
    if r.world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def finish(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def shard(n: int, r: Ranks) -> range:
    """Rank r's contiguous block of n units (the blocks cover 0..n-1 once,
    sizes differ by at most one)."""
    q, m = divmod(n, r.world)
    lo = r.rank * q + min(r.rank, m)
    return range(lo, lo + q + (1 if r.rank < m else 0))


def scene_seed(base: int, r: Ranks, stride: int = 1) -> int:
    """Seed of rank r's scenes: every rank simulates different scenes."""
    return base + stride * r.rank


def weak_rate(units_per_rank: float, ms_max: float, r: Ranks) -> float:
    """Whole-job throughput (units per second) of ranks that each processed
    units_per_rank, timed by the slowest rank."""
    return r.world * units_per_rank / (ms_max / 1e3)


def gather_rows(r: Ranks, a, device: str = "cuda"):
    """Every rank's block of rows of a (numpy, any row count, the same
    trailing shape and dtype on every rank), concatenated in rank order on
    every rank: with contiguous shards (shard()) that is the global order."""
    import numpy as np

    if r.world == 1:
        return a
    import torch
    import torch.distributed as dist

    a = np.ascontiguousarray(a)
    n = torch.tensor([a.shape[0]], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n) for _ in range(r.world)]
    dist.all_gather(sizes, n)
    sizes = [int(x.item()) for x in sizes]
    m = max(sizes)
    row = int(np.prod(a.shape[1:], dtype=np.int64)) if a.ndim > 1 else 1
    raw = a.view(np.uint8).reshape(a.shape[0], row * a.dtype.itemsize)
    buf = np.zeros((m, row * a.dtype.itemsize), dtype=np.uint8)
    buf[: a.shape[0]] = raw
    t = torch.from_numpy(buf).to(device)
    parts = [torch.empty_like(t) for _ in range(r.world)]
    dist.all_gather(parts, t)
    out = np.concatenate([p.cpu().numpy()[:k] for p, k in zip(parts, sizes)], axis=0)
    return out.reshape(-1).view(a.dtype).reshape((sum(sizes),) + a.shape[1:])


def members_of(n_members: int, r: Ranks) -> list[int]:
    """The ensemble members rank r trains and evaluates (round robin)."""
    return [q for q in range(n_members) if q % r.world == r.rank]
