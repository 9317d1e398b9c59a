"""Runs a few time steps of a named workload on cuda:0, for profilers.

    python -m rfsyn_b200.profile --workload c2 --steps 16 [--schedule fused|split] [--n N]
    python -m rfsyn_b200.profile --workload c3 --steps 16
    python -m rfsyn_b200.profile --workload c4 --steps 16 [--scenes S]

The scene (or the batch of scenes) is created and uploaded first, then
`steps` time steps are launched kernel by kernel and timed with CUDA events
per kernel group (sweep vs the rest).  --n rescales the C2 workload to an
n^3 grid (same recipe) for captures that must stay small.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import rfsyn_b200 as rb  # noqa: E402
from rfsyn_b200 import scenes  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--scenes", type=int, default=512)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--schedule", default="fused", choices=["fused", "split"])
    ap.add_argument("--n", type=int, default=0)
    args = ap.parse_args()
    if args.workload == "c4":
        ws = scenes.c4(seed=4, n_scenes=args.scenes)
        setups = [scenes.scene_setup(x) for x in ws]
        b = rb.Batch([scenes.run_config(x) for x in ws], [st.ptr if st else None for st in setups])
        bi = b.info()
        print(f"batch plan: rows {bi.tile_j}, ring {bi.ring_depth}, scenes {bi.scenes}, cells {bi.cells}", flush=True)
        sweep_ms, other_ms = b.time_kernels(args.steps)
        b.close()
        print(f"c4 x{args.scenes}: {args.steps} steps, sweep {sweep_ms / args.steps:.3f} ms/step, "
              f"other {other_ms / args.steps:.3f} ms/step")
        return
    if args.workload == "c3":
        w = scenes.c3()
        w.n_steps = max(args.steps, 1)
        setup = scenes.scene_setup(w)
        sim = rb.Sim(scenes.run_config(w), setup.ptr if setup else None, None)
        info = sim.info()
        print(f"plan: mode {info.tma}, rows {info.tile_j}, ring {info.ring_depth}, list cells {info.list_cells}",
              flush=True)
        sweep_ms, other_ms = sim.time_kernels(args.steps)
        sim.close()
        print(f"{w.name}: {args.steps} steps, sweep {sweep_ms / args.steps:.3f} ms/step, "
              f"other {other_ms / args.steps:.3f} ms/step")
        return
    w = scenes.c2() if args.workload == "c2" else scenes.c1(precision=rb.FP32)
    if args.n:
        w = scenes.scaled(w, args.n, max(args.steps, 8))
    w.schedule = rb.FUSED if args.schedule == "fused" else rb.SPLIT
    w.n_steps = max(args.steps, 1)
    setup = scenes.sphere_setup(w)
    sim = rb.Sim(scenes.run_config(w), setup.ptr if setup else None, None)
    info = sim.info()
    print(f"plan: mode {info.tma}, rows {info.tile_j}, ring {info.ring_depth}, segment {info.seg_len}, "
          f"interior items {info.interior_items}, edge items {info.edge_items}", flush=True)
    sweep_ms, other_ms = sim.time_kernels(args.steps)
    sim.close()
    print(f"{w.name}: {args.steps} steps, sweep {sweep_ms / args.steps:.3f} ms/step, "
          f"other {other_ms / args.steps:.3f} ms/step")


if __name__ == "__main__":
    main()
