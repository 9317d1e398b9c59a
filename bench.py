"""Benchmark of the FDTD stage time loop (one JSON line on rank 0).

Workload: the 256^3 FP32 scene with 24 subpixel-smoothed dielectric spheres,
3 Debye spheres, 12-cell CPML, 16 probes x 256 DFT bins and 4000 steps
(rfsyn_b200.scenes.c2).  A bench "step" is one full simulation of that scene
(reset + 4000 time steps, the probe spectra accumulating on the device as
the steps run).  Metric:
Mcell-updates/s = nx*ny*nz*n_steps*K / seconds, whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times rfsyn's own CPU loop (compiled from its sources into
oracle/_ref, or the CPU oracle port when that build is absent) on all host
cores, on a bounded sample of the same scene.

On one GPU the default run also runs the other workloads after its own
measurements -- the C3 periodic cell, the C4 batch of 512 scenes and the C5
surrogate path, each `python bench.py --workload cN ...` in its own process
-- and carries their figures under "other_workloads" (--no-other-workloads
skips them; about three minutes).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS = ROOT / "MEASURED_PEAKS.json"
TRAFFIC = ROOT / "profiles" / "sweep_queue_c2.md"
METRIC = "Mcell-updates/s"


SWEEP_KERNEL = {
    0: "k_sweep_interior + k_sweep_edge (one H+E sweep, cp.async ring)",
    1: "k_sweep_interior_tma + k_sweep_edge (one H+E sweep)",
    2: "k_sweep_q (one H+E sweep: interior + x-slab + edge launches)",
    3: "k_sweep_q (one H+E sweep: interior + x-slab + edge launches, shifted tiles)",
    4: "k_sweep_q (one H+E sweep: interior + x-slab + edge launches, narrow z-slab tiles)",
}


def hbm_peak() -> tuple[float, str]:
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_per_launch():
    """dram bytes (read + write) per sweep launch from the committed ncu
    summary (line 'traffic_bytes_per_launch: N'), or None."""
    try:
        for line in TRAFFIC.read_text().splitlines():
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                     f[5:9]):
                    if val.lower() == "active":
                        reasons.add(name)
        except Exception:
            pass
        finally:
            if self.path:
                try:
                    os.unlink(self.path)
                except OSError:
                    pass
        load = [v for v in sm if mx and v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes_per_sweep(info, esz: int) -> float:
    """Compulsory bytes of one H+E sweep launch: every field component read
    and written once (12 accesses per cell), the material code (1 B), and
    4 psi read + write per (cell, CPML slab axis); E of interface-list cells
    is written by the list kernel, not by the sweep."""
    b = info.cells * (12 * esz + 1) - info.list_cells * 3 * esz
    b += info.slab_cell_axes * 8 * esz
    return float(b)


# ---------------------------------------------------------------------------
# CPU reference arm
# ---------------------------------------------------------------------------
COPY_BYTES_PER_CELL = 170  # rfsyn's resident copy of a scene: 6 fields, 12 psi, materials, driver state


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def mem_available() -> int:
    try:
        for line in Path("/proc/meminfo").read_text().splitlines():
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except (OSError, ValueError):
        pass
    return 0


def cpu_copies(workload) -> int:
    """Independent copies run side by side: one per host core, as many as
    60 % of the available memory holds."""
    cores = os.cpu_count() or 1
    per = max(1, (workload.nx + 1) * (workload.ny + 1) * (workload.nz + 1) * COPY_BYTES_PER_CELL)
    avail = mem_available()
    return max(1, min(cores, int(0.6 * avail) // per if avail else cores))


def _cpu_worker(workload, steps, samples, warm, barrier, conn) -> None:
    """One process: builds rfsyn's copy of the scene, runs `warm` untimed
    steps (first touch of the calloc'd fields and psi), then `samples` timed
    samples of `steps` steps, each started together with the other copies."""
    import ctypes as C

    import oracle
    from tests.cases import workload_to_scene

    try:
        scene = workload_to_scene(workload)
        scene.probes, scene.freqs = [], []
        cs = scene.to_c()
        lib = C.CDLL(str(oracle.REF_LIB))
        lib.scn_bench_create.restype = C.c_void_p
        lib.scn_bench_create.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.scn_bench_steps.restype = C.c_int
        lib.scn_bench_steps.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_double)]
        lib.scn_bench_destroy.argtypes = [C.c_void_p]
        setup = C.c_double(0)
        h = lib.scn_bench_create(C.byref(cs), C.byref(setup))
        t = C.c_double(0)
        ok = bool(h) and lib.scn_bench_steps(h, warm, C.byref(t)) == 0
        times = []
        for _ in range(samples):
            barrier.wait()
            ok = ok and lib.scn_bench_steps(h, steps, C.byref(t)) == 0
            times.append(t.value)
        barrier.wait()
        lib.scn_bench_destroy(h)
        conn.send({"ok": ok, "setup_s": setup.value, "times": times})
    except Exception as exc:  # report, and keep the barrier going for the others
        barrier.abort()
        conn.send({"ok": False, "error": repr(exc)})


def cpu_reference(workload, steps: int, samples: int, copies: int | None = None, warm: int = 1) -> dict:
    """rfsyn's own CPU loop (oracle/_ref) on `copies` independent processes,
    each with its own copy of the scene: per sample every copy runs `steps`
    time steps after a common barrier; the sample's rate is all copies'
    cell-updates over the slowest copy's time.  Returns the median rate over
    the samples, the per-copy rate and the host it ran on.  Without the
    compiled reference, the oracle port times one copy."""
    import multiprocessing as mp

    import oracle

    model, cores = cpu_model(), os.cpu_count() or 1
    if not oracle.ref_available():
        from tests.cases import workload_to_scene

        scene = workload_to_scene(workload)
        scene.n_steps, scene.probes, scene.freqs = steps, [], []
        t0 = time.perf_counter()
        oracle.run_oracle(scene)
        loop = time.perf_counter() - t0
        v = workload.cells * steps / loop / 1e6
        return {"value": v, "unit": METRIC, "cores": 1, "kind": "port", "per_copy": v, "samples": [v],
                "cpu_model": model, "nproc": cores,
                "sample": f"1 copy of the {workload.nx}^3 scene x {steps} of its {workload.n_steps} steps (FP64)"}
    copies = copies or cpu_copies(workload)
    ctx = mp.get_context("spawn")  # never fork a process that holds a CUDA context
    barrier = ctx.Barrier(copies, timeout=1800)
    pipes = [ctx.Pipe(duplex=False) for _ in range(copies)]
    procs = [ctx.Process(target=_cpu_worker, args=(workload, steps, samples, warm, barrier, w), daemon=True)
             for (_, w) in pipes]
    for pr in procs:
        pr.start()
    res = [r.recv() for (r, _) in pipes]
    for pr in procs:
        pr.join()
    if not all(r.get("ok") for r in res):
        raise RuntimeError(f"reference CPU run failed: {[r.get('error') for r in res if not r.get('ok')]}")
    rates = [copies * workload.cells * steps / max(r["times"][s] for r in res) / 1e6 for s in range(samples)]
    value = statistics.median(rates)
    return {"value": value, "unit": METRIC, "cores": copies, "kind": "reference", "per_copy": value / copies,
            "samples": rates, "cpu_model": model, "nproc": cores,
            "setup_s": max(r["setup_s"] for r in res),
            "sample": (f"{copies} independent processes (one per core, of {cores}), each its own copy of the "
                       f"{workload.nx}^3 scene: {warm} untimed warm-up step, then {samples} samples of {steps} of "
                       f"its {workload.n_steps} steps started together (FP64; Debye spheres at their static "
                       f"permittivity; median sample)")}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from rfsyn_b200 import scenes

    w = scenes.c2()
    # one resident copy per process: the warm-up samples are the bench's
    # warm-up steps, the timed samples its steps
    cb = cpu_reference(w, args.ref_sample_steps, args.warmup + args.steps)
    rates = cb.pop("samples")[args.warmup:]
    value = statistics.median(rates)
    cb["value"], cb["per_copy"] = value, value / cb["cores"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG32 scene)",
        "config": {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "n_steps_sampled": args.ref_sample_steps,
                   "n_steps_full": w.n_steps},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def traced_call(fn):
    """Runs fn() with the library's phase trace on and its stderr lines
    captured; returns (fn's result, {phase: ms})."""
    import rfsyn_b200 as rb

    lib = rb.load()
    sys.stderr.flush()
    saved = os.dup(2)
    with tempfile.TemporaryFile(mode="w+b") as tmp:
        os.dup2(tmp.fileno(), 2)
        try:
            lib.fdtd_b200_apply_setting(b"trace", b"true")
            out = fn()
        finally:
            lib.fdtd_b200_apply_setting(b"trace", b"default")
            os.dup2(saved, 2)
            os.close(saved)
        tmp.seek(0)
        text = tmp.read().decode(errors="replace")
    phases = {}
    for line in text.splitlines():
        if line.startswith("rfsyn_b200 trace: ") and line.endswith(" ms"):
            name, ms = line[len("rfsyn_b200 trace: "):-3].rsplit(" ", 1)
            phases[name] = phases.get(name, 0.0) + float(ms)
    return out, phases


def fp64_reference_run(w, setup) -> dict:
    """The workload in FP64 on the device: one warm-up run, one timed run
    (CUDA events); returns its spectra and the loop's milliseconds."""
    import dataclasses

    import rfsyn_b200 as rb
    from rfsyn_b200 import scenes

    w64 = dataclasses.replace(w, precision=rb.FP64)
    sim = rb.Sim(scenes.run_config(w64), setup.ptr if setup else None, None)
    try:
        sim.advance(w64.n_steps)
        sim.reset()
        ms = sim.advance_timed(w64.n_steps)
        return {"dft": sim.dft(), "ms": ms}
    finally:
        sim.close()


def run_b200(args) -> None:
    import torch
    import rfsyn_b200 as rb
    from rfsyn_b200 import ranks, scenes

    rk = ranks.from_env()
    world, rank, local = rk.world, rk.rank, rk.local
    torch.cuda.set_device(local)
    ranks.init(rk, "nccl", 120)

    # each rank simulates its own independent scene (weak scaling, no collective on the data path)
    w = (scenes.c3(seed=ranks.scene_seed(3, rk)) if args.workload == "c3"
         else scenes.c2(seed=ranks.scene_seed(2, rk)))
    rc = scenes.run_config(w)
    setup = scenes.scene_setup(w)
    sim = rb.Sim(rc, setup.ptr if setup else None, None)
    stream = torch.cuda.ExternalStream(sim.stream)
    info = sim.info()
    esz = 4 if w.precision == rb.FP32 else 8

    def one_step():
        sim.reset()
        sim.advance(w.n_steps)

    for _ in range(args.warmup):
        one_step()
    sim.synchronize()
    lib = rb.load()
    launches0 = lib.fdtd_b200_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ranks.barrier(rk)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            one_step()
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    launches = lib.fdtd_b200_launch_count() - launches0
    ms = ranks.max_over(rk, start.elapsed_time(end))
    ranks.barrier(rk)
    clocks = clk.summary()
    value = ranks.weak_rate(w.cells * w.n_steps * args.steps, ms, rk) / 1e6

    # results of the last timed step: probes and spectra (correctness guard)
    dft = sim.dft()
    finite = bool(np.all(np.isfinite(dft)))

    # live per-kernel timing of the dominant sweep kernel (same scene)
    sim.reset()
    sweep_ms, other_ms = sim.time_kernels(200)
    sweep_launch_ms = sweep_ms / 200
    alg = algorithmic_bytes_per_sweep(info, esz)
    peak, peak_kind = hbm_peak()
    achieved = alg / (sweep_launch_ms / 1e3) / 1e9
    # the committed ncu capture covers the C2 scene's queue sweep only
    traffic = ncu_traffic_per_launch() if args.workload == "c2" and info.tma >= 2 else None
    sim.close()

    # end to end through the C ABI with host buffers: setup on the host,
    # scene upload, the full loop, DFT, download of series and spectra
    # every call with the library's phase trace on (a few lines to a file):
    # where each call spends its time
    calls = []
    h2d = d2h = 0

    def one_call():
        t0 = time.perf_counter()
        out = rb.run(rc, setup.ptr if setup else None, None)
        return out, (time.perf_counter() - t0) * 1e3

    for _ in range(max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        (r, call_ms), call_phases = traced_call(one_call)
        calls.append((call_ms, call_phases))
        d2h = r["td"].nbytes + r["dft"].nbytes
    h2d = info.h2d_bytes
    e2e_calls = [round(c[0], 1) for c in calls]
    e2e_mean = sum(c[0] for c in calls) / len(calls)
    # the median call: the host set-up of one call now and then takes far
    # longer than the others on a shared host (every call is listed beside,
    # with the phases of the median and of the slowest call)
    by_time = sorted(calls, key=lambda c: c[0])
    phases, slowest_phases = by_time[len(by_time) // 2][1], by_time[-1][1]
    e2e_ms = ranks.max_over(rk, statistics.median(c[0] for c in calls))
    e2e_value = ranks.weak_rate(w.cells * w.n_steps, e2e_ms, rk) / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "c2":
        try:
            cb = cpu_reference(w, args.ref_sample_steps, 3)
            cb.pop("samples", None)
            cpu = cb
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": 0, "kind": "unavailable", "sample": str(exc)}

    # accuracy of the measured FP32 run: the same scene in FP64 on the GPU
    # (bit-exact with rfsyn's double-precision loop wherever that runs),
    # timed as well for the like-for-like precision figure
    fp64 = fp64_reference_run(w, setup)
    err = np.linalg.norm(dft - fp64["dft"], axis=1) / np.linalg.norm(fp64["dft"], axis=1)
    parity = {"spec_l2_max": float(err.max()), "spec_l2_median": float(np.median(err)), "bound": 1e-4,
              "probes": int(err.size), "bins": int(dft.shape[1]),
              "vs": "fp64-gpu (the FP64 device loop: bit-exact with rfsyn's FP64 loop and the oracle at their sizes)"}

    ranks.finish(rk)
    if rank != 0:
        return
    # a default single-GPU run also records the other workloads (after this
    # workload's measurements, so they do not disturb them)
    others = other_workloads() if (world == 1 and args.workload == "c2" and not args.no_other_workloads) else None
    field_mb = (w.nx + 1) * (w.ny + 1) * (w.nz + 1) * esz / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": ("synthetic (seeded PCG32 scene: 24 smoothed + 3 Debye spheres)" if args.workload == "c2" else
                 "synthetic (seeded PCG32 cell: TF/SF plane wave, tilted 3x3 slab, 2-pole Lorentz layer)"),
        "config": {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "n_steps": w.n_steps, "npml": w.npml,
                   "probes": len(w.probes), "dft_bins": len(w.freqs), "spheres": len(w.spheres),
                   "list_cells": info.list_cells, "dispersive_samples": info.dispersive,
                   "schedule": "fused" if info.schedule == rb.FUSED else "split", "tile_j": info.tile_j,
                   "sweep_mode": {0: "cp.async", 1: "tma-interior", 2: "tma-queue", 3: "tma-queue-shifted",
                                  4: "tma-queue-narrow-z"}.get(info.tma),
                   "ring_depth": info.ring_depth, "single_queue": bool(info.unified),
                   "seg_len": info.seg_len, "seg_edge": info.seg_edge, "two_rows_ring": info.interior_ring2,
                   "plan": f"{info.tile_j},{info.ring_depth},{info.seg_len},{info.seg_edge},{info.tma},"
                           f"{info.unified},{info.interior_ring2}",
                   "parallelism": f"scene-replicas x{world}",
                   "l2": f"inputs larger than L2 (fields 6 x 2 x {field_mb:.0f} MB per scene)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind, "kernel": SWEEP_KERNEL.get(info.tma, "k_h_split + k_e_split"),
                     "algorithmic_bytes_per_launch": alg, "launch_ms": sweep_launch_ms,
                     "other_kernels_ms_per_step": other_ms / 200},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms, "statistic": "median of the calls", "calls": len(e2e_calls),
                "calls_ms": e2e_calls, "mean_ms": e2e_mean,
                "slowest_call_phases_ms": {k: round(v, 3) for k, v in slowest_phases.items()},
                "phases_ms": {k: round(v, 3) for k, v in phases.items()}},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "finite": finite,
        "parity": parity,
        "fp64": {"value": w.cells * w.n_steps / (fp64["ms"] / 1e3) / 1e6, "unit": METRIC, "ms_per_step": fp64["ms"],
                 "note": "the same scene and step loop in FP64 on the device, one run after a warm-up run"},
    }
    if others is not None:
        line["other_workloads"] = others
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# The other workloads, summarised in the default run's line
# ---------------------------------------------------------------------------
OTHER_RUNS = {
    "c3": ["--workload", "c3", "--steps", "2", "--warmup", "3", "--no-cpu-baseline"],
    "c4": ["--workload", "c4", "--steps", "2", "--warmup", "3"],
    "c5": ["--workload", "c5"],
}


def _summary(name: str, d: dict) -> dict:
    """The figures of another workload's line that the default line carries."""
    r, e = d.get("roofline") or {}, d.get("e2e") or {}
    out = {"metric": d.get("metric"), "value": d.get("value"), "unit": d.get("unit"),
           "ms_per_step": d.get("ms_per_step"), "frac": r.get("frac"), "e2e": e.get("value"),
           "clocks": d.get("clocks")}
    if name == "c3":
        out.update({"workload": (d.get("config") or {}).get("workload"), "plan": (d.get("config") or {}).get("plan"),
                    "parity_spec_l2_max": (d.get("parity") or {}).get("spec_l2_max"),
                    "fp64": (d.get("fp64") or {}).get("value")})
    elif name == "c4":
        out.update({"scenes_per_s": d.get("scenes_per_s"), "plain_one_at_a_time": d.get("plain_one_at_a_time")})
    elif name == "c5":
        out.update({"speedup_vs_plain": d.get("speedup_vs_plain"), "accepted_scene_frac": d.get("accepted_scene_frac"),
                    "plain_one_at_a_time_scenes_s": d.get("plain_one_at_a_time_scenes_s"),
                    "batched_fdtd_scenes_s": d.get("batched_fdtd_scenes_s"),
                    "transfer_rel_err": d.get("transfer_rel_err"), "timings_s": d.get("timings_s")})
    return out


def other_workloads() -> dict:
    """Runs the C3, C4 and C5 benches (each its own process, one after the
    other on this GPU) and returns their figures, so a default single-GPU
    run records every workload; a workload that fails is reported, never
    fatal."""
    # each run is a standalone single-GPU process (no rendezvous variables)
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE", "GROUP_RANK", "MASTER_ADDR",
                        "MASTER_PORT") and not k.startswith("TORCHELASTIC_")}
    res = {}
    for name, argv in OTHER_RUNS.items():
        t0 = time.perf_counter()
        try:
            p = subprocess.run([sys.executable, str(ROOT / "bench.py"), *argv], capture_output=True, text=True,
                               timeout=1200, env=env)
            lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
            if p.returncode != 0 or not lines:
                res[name] = {"error": f"exit {p.returncode}: {(p.stderr or p.stdout)[-300:]}"}
            else:
                res[name] = _summary(name, json.loads(lines[-1]))
        except Exception as exc:  # reported, never fatal
            res[name] = {"error": str(exc)[:300]}
        res[name]["wall_s"] = round(time.perf_counter() - t0, 1)
        res[name]["command"] = "python bench.py " + " ".join(argv)
    return res


# ---------------------------------------------------------------------------
# Batched scenes (--workload c4)
# ---------------------------------------------------------------------------
def run_batch(args) -> None:
    """512 independent uneven scenes (rfsyn_b200.scenes.c4) advanced together
    by one batch: a step = one full run of every scene (reset + 1500 time
    steps).  Metric Mcell-updates/s over the whole batch; scenes/s beside it,
    with the plain one-scene-at-a-time GPU session timed on a sample of the
    same scenes as the baseline the batch is measured against."""
    import torch

    import rfsyn_b200 as rb
    from rfsyn_b200 import ranks, scenes

    rk = ranks.from_env()
    world, rank, local = rk.world, rk.rank, rk.local
    torch.cuda.set_device(local)
    ranks.init(rk, "nccl", 300)
    # one set of args.scenes scenes, each rank batching its contiguous shard
    # (strong scaling: the job's work is fixed as ranks are added)
    ws_all = scenes.c4(seed=4, n_scenes=args.scenes)
    ws = [ws_all[q] for q in ranks.shard(len(ws_all), rk)]
    n_steps = ws[0].n_steps
    cells = sum(w.cells for w in ws)
    setups = [scenes.scene_setup(w) for w in ws]
    rcs = [scenes.run_config(w) for w in ws]
    t0 = time.perf_counter()
    b = rb.Batch(rcs, [s.ptr if s else None for s in setups])
    create_s = time.perf_counter() - t0
    info = b.info()
    stream = torch.cuda.ExternalStream(b.stream)

    def one_step():
        b.reset()
        b.advance(n_steps)

    for _ in range(args.warmup):
        one_step()
    b.synchronize()
    lib = rb.load()
    launches0 = lib.fdtd_b200_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ranks.barrier(rk)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            one_step()
        end.record(stream)
        end.synchronize()
    b.synchronize()
    launches = lib.fdtd_b200_launch_count() - launches0
    ms = ranks.max_over(rk, start.elapsed_time(end))
    clocks = clk.summary()
    # the ranks' shards partition the set: the whole job's cells are summed
    cells_all = ranks.sum_over(rk, float(cells))
    value = cells_all * n_steps * args.steps / (ms / 1e3) / 1e6
    scenes_s = len(ws_all) * args.steps / (ms / 1e3)
    finite = all(bool(np.all(np.isfinite(b.dft(q)))) for q in range(0, len(ws), max(1, len(ws) // 16)))
    # sweep kernels alone (CUDA events around the sweep launches of each step)
    b.reset()
    sw, ot = b.time_kernels(50)
    b.close()

    # plain one-scene-at-a-time GPU sessions on a sample of the same scenes
    sample = ws[: args.plain_sample]
    plain_ms = 0.0
    for w, st in zip(sample, setups):
        sim = rb.Sim(scenes.run_config(w), st.ptr if st else None, None)
        sim.advance(n_steps)          # warm (graph build)
        sim.reset()
        plain_ms += sim.advance_timed(n_steps)
        sim.close()
    plain_scenes_s = len(sample) / (plain_ms / 1e3)

    # end to end: scene set-up and upload, the full run, every probe series
    # and spectrum back on the host
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b2 = rb.Batch(rcs, [s.ptr if s else None for s in setups])
    b2.advance(n_steps)
    d2h = 0
    for q in range(len(ws)):
        d2h += b2.probes(q).nbytes + b2.dft(q).nbytes
    e2e_ms = ranks.max_over(rk, (time.perf_counter() - t0) * 1e3)
    b2.close()
    ranks.finish(rk)
    if rank != 0:
        return
    esz = 4
    alg = cells * (12 * esz + 1) + info.slab_cell_axes * 8 * esz
    peak, peak_kind = hbm_peak()
    sweep_launch_ms = sw / 50
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded PCG32 scenes: 0-6 spheres / boxes each)",
        "config": {"workload": f"c4_batch{len(ws_all)}_32to96_fp32", "scenes": len(ws_all),
                   "scenes_per_rank": len(ws), "cells": int(cells_all),
                   "n_steps": n_steps, "npml": 8, "probes_per_scene": 4, "dft_bins": 128,
                   "plan": {"tile_j": info.tile_j, "ring_depth": info.ring_depth, "mode": info.mode,
                            "seg_interior": info.seg_interior, "seg_edge": info.seg_edge,
                            "single_queue": bool(info.unified)},
                   "items": [info.items_interior, info.items_xslab, info.items_edge],
                   "parallelism": f"scene shards x{world}", "l2": "inputs larger than L2 (fields 12 x 4 B x 130 M cells)"},
        "scenes_per_s": scenes_s,
        "plain_one_at_a_time": {"scenes_per_s": plain_scenes_s, "sample": len(sample),
                                "speedup_batched": scenes_s / world / plain_scenes_s},
        "roofline": {"bound": "hbm", "achieved": alg / (sweep_launch_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (sweep_launch_ms / 1e3) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                     "kernel": "k_sweep_qb (one batched H+E sweep: interior + x-slab + edge launches)",
                     "algorithmic_bytes_per_launch": alg, "launch_ms": sweep_launch_ms,
                     "other_kernels_ms_per_step": ot / 50},
        "e2e": {"value": cells_all * n_steps / (e2e_ms / 1e3) / 1e6, "unit": METRIC, "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "includes": "scene set-up and upload"},
        "create_s": create_s,
        "gpu_launches": int(launches), "launches_per_time_step": info.launches_per_step,
        "clocks": clocks, "finite": finite,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Surrogate (--workload c5)
# ---------------------------------------------------------------------------
def run_surrogate(args) -> None:
    """Transfer-function surrogate: training data from the batched FDTD
    (48^3 scenes at dx 2 mm, 0-8 spheres, 1 tx + 4 rx each, 1500 steps), a
    5-member ensemble of 54 -> 512 x 4 (GELU) -> 512 MLPs trained on the GPU
    (20k Adam steps, batch 256, lr 1e-3 cosine), held-out scenes answered by
    the ensemble where its spread is <= 2 % of the norm and by the batched
    FDTD otherwise.  Metric: held-out scenes/s of that path (wall clock, the
    ensemble's inference plus the fallback FDTD runs), beside the plain
    one-scene-at-a-time GPU FDTD and the transfer-function error.  With
    several ranks the scene sets are sharded (each rank runs its block of
    scenes, the rows are gathered on every rank), the members split over
    the ranks and their predictions gathered; times are the slowest rank's."""
    import torch

    import rfsyn_b200 as rb
    from rfsyn_b200 import ranks, scenes
    from rfsyn_b200 import surrogate as sg

    rk = ranks.from_env()
    torch.cuda.set_device(rk.local)
    ranks.init(rk, "nccl", 1800)
    ws_tr = sg.c5_scenes(seed=51, n_scenes=args.train_scenes)
    ws_te = sg.c5_scenes(seed=52, n_scenes=args.test_scenes)
    tm = {}
    ranks.barrier(rk)
    t0 = time.perf_counter()
    X_tr, H_tr = sg.sharded_transfer_functions(ws_tr, rk, timings=tm)
    gen_s = ranks.max_over(rk, time.perf_counter() - t0)
    G_tr = sg.scene_transfer_targets(ws_tr, H_tr)
    sur = sg.Surrogate(members=5, width=512, depth=4, seed=3, r=rk)
    t0 = time.perf_counter()
    losses = sur.fit(X_tr, G_tr, steps=args.train_steps, batch=256, lr=1e-3)
    train_s = ranks.max_over(rk, time.perf_counter() - t0)
    # held-out truth from the batched FDTD (also its throughput)
    tm_te = {}
    t0 = time.perf_counter()
    X_te, H_te = sg.sharded_transfer_functions(ws_te, rk, timings=tm_te)
    fdtd_batched_wall = ranks.max_over(rk, time.perf_counter() - t0)
    fdtd_batched_scenes_s = len(ws_te) / (ranks.max_over(rk, tm_te.get("fdtd_ms", 0.0)) / 1e3)
    pred = sur.predict(ws_te, X_te)
    err_all = sg.rel_err(pred.H, H_te)
    # the surrogate path with fallback, wall clock end to end
    torch.cuda.synchronize()
    ranks.barrier(rk)
    t0 = time.perf_counter()
    res = sg.infer_with_fallback(sur, ws_te, threshold=args.threshold)
    path_s = ranks.max_over(rk, time.perf_counter() - t0)
    err = sg.rel_err(res["H"], H_te)
    fell = set(res["fallback"])
    acc_rows = np.asarray([q not in fell for q in range(len(ws_te)) for _ in range(4)])
    # plain one-scene-at-a-time GPU FDTD on a sample (rank 0's GPU)
    plain_scenes_s = None
    if rk.rank == 0:
        plain_ms = 0.0
        sample = ws_te[: args.plain_sample]
        for w in sample:
            st = scenes.scene_setup(w)
            sim = rb.Sim(scenes.run_config(w), st.ptr if st else None, None)
            sim.advance(w.n_steps)
            sim.reset()
            plain_ms += sim.advance_timed(w.n_steps)
            sim.close()
        plain_scenes_s = len(sample) / (plain_ms / 1e3)
    sur.close()
    ranks.finish(rk)
    if rk.rank != 0:
        return
    value = len(ws_te) / path_s
    line = {
        "metric": "scenes/s (batched FDTD + surrogate, held-out)", "value": value, "unit": "scenes/s",
        "n_gpus": rk.world, "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "bf16 GEMMs / fp32 FDTD", "data": "synthetic (seeded PCG32 scenes)",
        "config": {"workload": "c5_surrogate_48cube_dx2mm", "train_scenes": len(ws_tr), "test_scenes": len(ws_te),
                   "samples_per_scene": 4, "members": 5, "net": "54-512x4(GELU)-512", "train_steps": args.train_steps,
                   "batch": 256, "lr": 1e-3, "threshold": args.threshold, "bins": sg.N_BINS,
                   "parallelism": f"scene shards + ensemble members x{rk.world}"},
        "plain_one_at_a_time_scenes_s": plain_scenes_s, "speedup_vs_plain": value / plain_scenes_s,
        "batched_fdtd_scenes_s": fdtd_batched_scenes_s,
        "accepted_scene_frac": 1.0 - len(fell) / len(ws_te),
        "transfer_rel_err": {"final_median": float(np.median(err)), "final_p95": float(np.percentile(err, 95)),
                             "final_max": float(err.max()),
                             "accepted_median": float(np.median(err[acc_rows])) if acc_rows.any() else None,
                             "accepted_p95": float(np.percentile(err[acc_rows], 95)) if acc_rows.any() else None,
                             "network_only_median": float(np.median(err_all)),
                             "network_only_p95": float(np.percentile(err_all, 95))},
        "timings_s": {"data_generation": gen_s, "data_generation_device": tm.get("fdtd_ms", 0.0) / 1e3,
                      "training": train_s, "path_surrogate": res["surrogate_s"], "path_fallback_fdtd": res["fdtd_s"],
                      "heldout_fdtd_wall": fdtd_batched_wall},
        "final_train_losses": losses,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Profiling runs (--profile-steps N): a few steps launched kernel by kernel
# ---------------------------------------------------------------------------
def run_profile(args) -> None:
    """Creates the workload's scene (or batch) on cuda:0, then launches
    `--profile-steps` time steps kernel by kernel with CUDA events around the
    sweep and the rest, for profilers (ncu); prints the plan and the times.
    --n rescales the C2 recipe to an n^3 grid for captures that must stay
    small."""
    import rfsyn_b200 as rb
    from rfsyn_b200 import scenes

    steps = max(1, args.profile_steps)
    if args.workload == "c4":
        ws = scenes.c4(seed=4, n_scenes=args.scenes)
        setups = [scenes.scene_setup(x) for x in ws]
        b = rb.Batch([scenes.run_config(x) for x in ws], [st.ptr if st else None for st in setups])
        bi = b.info()
        print(f"batch plan: rows {bi.tile_j}, ring {bi.ring_depth}, scenes {bi.scenes}, cells {bi.cells}", flush=True)
        sweep_ms, other_ms = b.time_kernels(steps)
        b.close()
        print(f"c4 x{args.scenes}: {steps} steps, sweep {sweep_ms / steps:.3f} ms/step, other {other_ms / steps:.3f} ms/step")
        return
    if args.workload == "c3":
        w = scenes.c3()
    elif args.workload == "c1":
        w = scenes.c1(precision=rb.FP32)
    else:
        w = scenes.c2()
        if args.n:
            w = scenes.scaled(w, args.n, max(steps, 8))
    w.schedule = rb.FUSED if args.schedule == "fused" else rb.SPLIT
    w.n_steps = steps
    setup = scenes.scene_setup(w)
    sim = rb.Sim(scenes.run_config(w), setup.ptr if setup else None, None)
    info = sim.info()
    print(f"plan: {info.tile_j},{info.ring_depth},{info.seg_len},{info.seg_edge},{info.tma},{info.unified},"
          f"{info.interior_ring2} (rows, ring, interior / edge segments, mode, single queue, two-rows ring); "
          f"interior items {info.interior_items}, edge items {info.edge_items}, list cells {info.list_cells}",
          flush=True)
    sweep_ms, other_ms = sim.time_kernels(steps)
    sim.close()
    print(f"{w.name}: {steps} steps, sweep {sweep_ms / steps:.3f} ms/step, other {other_ms / steps:.3f} ms/step")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5, help="end-to-end calls, their median is e2e")
    ap.add_argument("--ref-sample-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-other-workloads", action="store_true",
                    help="c2 on one GPU: skip the C3, C4 and C5 runs summarised in the line")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--train-scenes", type=int, default=5000, help="c5: training scenes (4 samples each)")
    ap.add_argument("--test-scenes", type=int, default=500, help="c5: held-out scenes")
    ap.add_argument("--train-steps", type=int, default=20000, help="c5: Adam steps per member")
    ap.add_argument("--threshold", type=float, default=0.02, help="c5: ensemble spread that triggers FDTD")
    ap.add_argument("--scenes", type=int, default=512, help="c4: scenes per batch")
    ap.add_argument("--plain-sample", type=int, default=16, help="c4: scenes timed one at a time")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="profiling run: create the scene, launch this many steps kernel by kernel, print times")
    ap.add_argument("--n", type=int, default=0, help="profiling run, c2: rescale the recipe to an n^3 grid")
    ap.add_argument("--schedule", default="fused", choices=["fused", "split"], help="profiling run: schedule")
    args = ap.parse_args()
    if args.profile_steps:
        run_profile(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c4":
        run_batch(args)
    elif args.workload == "c5":
        run_surrogate(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
