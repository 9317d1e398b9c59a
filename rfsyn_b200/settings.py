"""rfsyn's pipeline config surface for the FDTD stage, and its GPU section.

rfsyn's job runner (cli/main.c:297-420, cmd_start) loads config.json and,
for every example i, builds the transform chain FDTD stage -> AWGN
(cli/settings.c:35-78) from the "fdtd" and "awgn" sections through
config.c's typed getters (cli/config.c:108-143) with the defaults of
cli/presets.h:14-29; the chain's output is written as example_%06d.iq.
This module reads the same keys with the same acceptance rules, so one
config.json gives the same fdtd_sim_config_t (build_fdtd_config), and adds
the "gpu.<name>" keys of the "fdtd" section, which rfsyn's own
`config set fdtd.gpu.<name> <value>` stores there (cli/main.c:233-290):

  process-wide (applied through fdtd_b200_apply_setting):
    gpu.precision  "fp32" | "fp64"     gpu.schedule  "fused" | "split"
    gpu.plan       "auto" | "tj,ns,seg_interior,seg_edge[,mode[,single_queue[,two_rows_ring]]]"
    gpu.tune       bool                gpu.trace     bool
  per run (read by run_examples):
    gpu.batch       examples simulated together in one batch (default 1)
    gpu.dft_bins, gpu.dft_f_lo_hz, gpu.dft_f_hi_hz
                    a running DFT of the probe at dft_bins frequencies
                    spaced linearly over [f_lo, f_hi] (default none)
    gpu.scene_seed  per-example scenes: example i gets 0-6 scatterers drawn
                    from PCG32(scene_seed, i) (rfsyn simulates the same empty
                    grid for every example; without the key so does this)

Unknown "gpu.*" keys are errors (a typo must not pass silently); rfsyn's own
keys keep rfsyn's rule (a missing or mistyped value falls back to the
preset).
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass

import numpy as np

from . import FIELD_EZ, SRC_SOFT, WAVE_GAUSSIAN_DERIV, FdtdSimConfig, dt_of, load as load_lib, last_error
from .scenes import Pcg32, Workload, draw_scatterers

# cli/presets.h:6-29 (the values rfsyn's getters fall back to)
PRESET = {
    ("job", "count"): 100, ("job", "n_samples"): 1024, ("job", "output_dir"): "output",
    ("awgn", "enabled"): 1, ("awgn", "snr_db"): 15.0, ("awgn", "seed"): 42,
    ("fdtd", "enabled"): 1, ("fdtd", "nx"): 50, ("fdtd", "ny"): 50, ("fdtd", "nz"): 50, ("fdtd", "dx"): 1e-3,
    ("fdtd", "courant"): 0.99, ("fdtd", "n_steps"): 200, ("fdtd", "npml"): 8,
    ("fdtd", "src_i"): -1, ("fdtd", "src_j"): -1, ("fdtd", "src_k"): -1,
    ("fdtd", "probe_i"): -1, ("fdtd", "probe_j"): -1, ("fdtd", "probe_k"): -1,
    ("fdtd", "t0"): 40.0, ("fdtd", "tau"): 8.0,
}

PROCESS_KEYS = ("precision", "schedule", "plan", "tune", "trace")
RUN_KEYS = ("batch", "dft_bins", "dft_f_lo_hz", "dft_f_hi_hz", "scene_seed")
LONG_MIN, LONG_MAX = -(1 << 63), (1 << 63) - 1
SIZE_MOD = 1 << 64


def _first_wins(pairs):
    """JSON object with the first of duplicate keys kept, as cJSON's lookup
    (the first matching child) sees it."""
    out = {}
    for k, v in pairs:
        out.setdefault(k, v)
    return out


def _no_constant(name):
    raise ValueError(f"config: {name} is not JSON")


def load(path: str | os.PathLike) -> dict:
    """config.json as a dict (config_load, cli/config.c:24-60); raises
    ValueError where rfsyn's parser refuses the text (NaN and Infinity
    included).  One difference, loud rather than silent: number literals
    that JSON forbids but cJSON hands to strtod (leading zeros, a trailing
    point, "-.5") are read by rfsyn and refused here.  Files written by
    rfsyn's `config set` (cJSON_Print) never hold them."""
    with open(path, "rb") as f:
        return json.loads(f.read().decode("utf-8"), object_pairs_hook=_first_wins, parse_constant=_no_constant)


def _item(cfg, section, key):
    s = cfg.get(section) if isinstance(cfg, dict) else None
    if not isinstance(s, dict):
        return None
    return s.get(key)


def _is_number(v) -> bool:
    return isinstance(v, (int, float)) and not isinstance(v, bool)


def get(cfg, section: str, key: str):
    """config_get: the value when it is a string, else None."""
    v = _item(cfg, section, key)
    return v if isinstance(v, str) else None


def _as_double(v) -> float:
    """A JSON number as cJSON's strtod reads it (integer literals beyond the
    double range become +-inf, as Python's float() would refuse)."""
    try:
        return float(v)
    except OverflowError:
        return math.inf if v > 0 else -math.inf


def get_double(cfg, section: str, key: str, default: float) -> float:
    """config_get_double: a JSON number, else the default."""
    v = _item(cfg, section, key)
    return _as_double(v) if _is_number(v) else default


def get_long(cfg, section: str, key: str, default: int) -> int:
    """config_get_long: a JSON number whose double value is finite, integral
    and within long's range, else the default."""
    v = _item(cfg, section, key)
    if not _is_number(v):
        return default
    d = _as_double(v)
    if not math.isfinite(d) or d != math.floor(d) or d < float(LONG_MIN) or d > float(LONG_MAX):
        return default
    if d == 2.0 ** 63:
        # passes the range check ((double)LONG_MAX rounds up to 2^63); the
        # C conversion of 2^63 to long gives LONG_MIN on x86-64
        return LONG_MIN
    return int(d)


def get_bool(cfg, section: str, key: str, default: int) -> int:
    """config_get_bool: a JSON true / false, else the default."""
    v = _item(cfg, section, key)
    return int(v) if isinstance(v, bool) else default


def _size_t(v: int) -> int:
    return v % SIZE_MOD


def build_fdtd_config(cfg) -> FdtdSimConfig:
    """The stage's fdtd_sim_config_t from the "fdtd" section
    (build_fdtd_config, cli/settings.c:6-33): sizes as size_t casts of the
    longs, source at the centre and probe at the centre + (6, 0, 0) when
    their indices are negative, Ez source and probe."""
    s = FdtdSimConfig()
    P = lambda k: PRESET[("fdtd", k)]
    s.nx = _size_t(get_long(cfg, "fdtd", "nx", P("nx")))
    s.ny = _size_t(get_long(cfg, "fdtd", "ny", P("ny")))
    s.nz = _size_t(get_long(cfg, "fdtd", "nz", P("nz")))
    s.dx = get_double(cfg, "fdtd", "dx", P("dx"))
    s.courant_safety = get_double(cfg, "fdtd", "courant", P("courant"))
    s.n_steps = _size_t(get_long(cfg, "fdtd", "n_steps", P("n_steps")))
    s.npml = _size_t(get_long(cfg, "fdtd", "npml", P("npml")))
    s.t0_over_dt = get_double(cfg, "fdtd", "t0", P("t0"))
    s.tau_over_dt = get_double(cfg, "fdtd", "tau", P("tau"))
    s.src_component = FIELD_EZ
    s.probe_component = FIELD_EZ
    si, sj, sk = (get_long(cfg, "fdtd", k, P(k)) for k in ("src_i", "src_j", "src_k"))
    s.src_i = s.nx // 2 if si < 0 else _size_t(si)
    s.src_j = s.ny // 2 if sj < 0 else _size_t(sj)
    s.src_k = s.nz // 2 if sk < 0 else _size_t(sk)
    pi, pj, pk = (get_long(cfg, "fdtd", k, P(k)) for k in ("probe_i", "probe_j", "probe_k"))
    s.probe_i = _size_t(s.nx // 2 + 6) if pi < 0 else _size_t(pi)
    s.probe_j = s.ny // 2 if pj < 0 else _size_t(pj)
    s.probe_k = s.nz // 2 if pk < 0 else _size_t(pk)
    return s


def setting_text(v) -> str:
    """A config value as the text fdtd_b200_apply_setting takes: strings as
    they are, booleans as true / false, integral numbers without a point."""
    if isinstance(v, bool):
        return "true" if v else "false"
    if _is_number(v):
        f = float(v)
        return str(int(f)) if math.isfinite(f) and f == math.floor(f) and abs(f) < 2 ** 63 else repr(f)
    if isinstance(v, str):
        return v
    raise ValueError(f"setting value {v!r} is not a string, number or boolean")


def _gpu_items(cfg):
    s = cfg.get("fdtd") if isinstance(cfg, dict) else None
    if not isinstance(s, dict):
        return []
    out = []
    for k, v in s.items():
        if k.startswith("gpu."):
            name = k[4:]
            if name not in PROCESS_KEYS and name not in RUN_KEYS:
                raise ValueError(f"unknown setting fdtd.{k}")
            out.append((name, v))
    return out


def apply_setting(name: str, value: str) -> None:
    if load_lib().fdtd_b200_apply_setting(name.encode(), value.encode()) != 0:
        raise ValueError(last_error())


def get_setting(name: str) -> str:
    import ctypes as C

    buf = C.create_string_buffer(128)
    if load_lib().fdtd_b200_get_setting(name.encode(), buf, len(buf)) != 0:
        raise ValueError(last_error())
    return buf.value.decode()


def apply_gpu_settings(cfg) -> None:
    """Applies the process-wide fdtd.gpu.* keys (precision, schedule, plan,
    tune, trace); raises ValueError naming the first one refused."""
    for name, v in _gpu_items(cfg):
        if name in PROCESS_KEYS:
            apply_setting(f"fdtd.gpu.{name}", setting_text(v))


@dataclass(frozen=True)
class RunOptions:
    batch: int = 1
    dft_bins: int = 0
    dft_f_lo_hz: float = 0.0
    dft_f_hi_hz: float = 0.0
    scene_seed: int | None = None

    def freqs(self) -> list:
        if not self.dft_bins:
            return []
        return list(np.linspace(self.dft_f_lo_hz, self.dft_f_hi_hz, self.dft_bins))


def run_options(cfg) -> RunOptions:
    """The per-run fdtd.gpu.* keys, validated."""
    vals = dict(_gpu_items(cfg))

    def integer(name, lo, default):
        if name not in vals:
            return default
        v = vals[name]
        if not _is_number(v) or float(v) != math.floor(float(v)) or v < lo:
            raise ValueError(f"fdtd.gpu.{name} must be an integer >= {lo}, got {v!r}")
        return int(v)

    def real(name, default):
        if name not in vals:
            return default
        v = vals[name]
        if not _is_number(v) or not math.isfinite(float(v)) or v < 0:
            raise ValueError(f"fdtd.gpu.{name} must be a finite number >= 0, got {v!r}")
        return float(v)

    o = RunOptions(batch=integer("batch", 1, 1), dft_bins=integer("dft_bins", 0, 0),
                   dft_f_lo_hz=real("dft_f_lo_hz", 0.0), dft_f_hi_hz=real("dft_f_hi_hz", 0.0),
                   scene_seed=integer("scene_seed", 0, None))
    if o.dft_bins and not o.dft_f_hi_hz >= o.dft_f_lo_hz:
        raise ValueError("fdtd.gpu.dft_f_hi_hz must not be below fdtd.gpu.dft_f_lo_hz")
    return o


def example_workload(cfg, index: int, opts: RunOptions | None = None) -> Workload:
    """Example `index` as a Workload: the stage's grid, CPML, source and probe
    exactly as fdtd_simulate_echo builds them (soft Gaussian-derivative Ez
    source of amplitude 1 with t0 and tau in steps, rfsyn's default CPML
    grading, one probe), the process's precision and schedule, the DFT bins
    and, with gpu.scene_seed, the example's own scatterers.  Raises
    ValueError where rfsyn's stage would fail (no steps, a grid the solver
    refuses, a source or probe outside the grid)."""
    from . import FP32, SPLIT

    opts = opts or run_options(cfg)
    s = build_fdtd_config(cfg)
    if s.n_steps == 0 or s.n_steps >= 1 << 40:
        raise ValueError("fdtd.n_steps must be positive")
    if not (1 <= s.nx <= 60000 and 1 <= s.ny <= 60000 and 1 <= s.nz <= 60000):
        raise ValueError("grid sizes must be within 1..60000")
    if not (s.dx > 0 and math.isfinite(s.dx) and 0 < s.courant_safety <= 1):
        raise ValueError("fdtd.dx must be positive and fdtd.courant in (0, 1]")
    if s.src_i > s.nx or s.src_j > s.ny or s.src_k > s.nz or s.probe_i > s.nx or s.probe_j > s.ny \
            or s.probe_k > s.nz:
        raise ValueError("source or probe outside the grid")
    dt = dt_of(s.dx, s.courant_safety)
    boxes, spheres = [], []
    if opts.scene_seed is not None:
        dims = (int(s.nx), int(s.ny), int(s.nz))
        if min(dims) < 2 * s.npml + 12:
            raise ValueError("fdtd.gpu.scene_seed needs every axis >= 2 npml + 12 cells")
        boxes, spheres = draw_scatterers(Pcg32(opts.scene_seed, index), dims, int(s.npml))
    return Workload(
        name=f"example_{index:06d}", nx=int(s.nx), ny=int(s.ny), nz=int(s.nz), dx=s.dx, n_steps=int(s.n_steps),
        npml=int(s.npml), courant=s.courant_safety,
        precision=FP32 if get_setting("precision") == "fp32" else 0,
        schedule=SPLIT if get_setting("schedule") == "split" else 1,
        sources=[dict(i=int(s.src_i), j=int(s.src_j), k=int(s.src_k), component=FIELD_EZ, mode=SRC_SOFT,
                      amplitude=1.0, waveform=WAVE_GAUSSIAN_DERIV, p0=s.t0_over_dt * dt, p1=s.tau_over_dt * dt,
                      p2=1.0)],
        probes=[dict(i=int(s.probe_i), j=int(s.probe_j), k=int(s.probe_k), component=FIELD_EZ)],
        freqs=opts.freqs(), boxes=boxes, spheres=spheres)


def awgn_of(cfg, index: int):
    """The AWGN stage's (snr_db as float, seed, stream) for example `index`,
    or None when the stage is off (cli/settings.c:60-73: awgn_create((float)
    snr_db, (uint64_t)seed, example_index))."""
    if not get_bool(cfg, "awgn", "enabled", PRESET[("awgn", "enabled")]):
        return None
    snr = float(np.float32(get_double(cfg, "awgn", "snr_db", PRESET[("awgn", "snr_db")])))
    seed = get_long(cfg, "awgn", "seed", PRESET[("awgn", "seed")]) % SIZE_MOD
    return snr, seed, index


def run_examples(cfg, indices) -> list:
    """The chain's output for each example index: the FDTD stage's probe
    series as complex64 (real part (float) of the FP64/FP32 series, as
    cli/fdtd_stage.c:20-21 stores it) followed, when awgn.enabled, by the
    AWGN stage with the example's stream, computed on the GPU.  Examples run
    gpu.batch at a time through the batch engine (one at a time by default).
    The fdtd section must be enabled."""
    from . import Batch, Sim
    from .scenes import run_config, scene_setup

    if not get_bool(cfg, "fdtd", "enabled", PRESET[("fdtd", "enabled")]):
        raise ValueError("fdtd.enabled is false: there is no FDTD stage to run")
    apply_gpu_settings(cfg)
    opts = run_options(cfg)
    indices = list(indices)
    out = []
    for c0 in range(0, len(indices), opts.batch):
        chunk = indices[c0:c0 + opts.batch]
        ws = [example_workload(cfg, i, opts) for i in chunk]
        noise = [awgn_of(cfg, i) for i in chunk]
        setups = [scene_setup(w) for w in ws]
        if len(chunk) == 1:
            sim = Sim(run_config(ws[0]), setups[0].ptr if setups[0] else None, None)
            try:
                sim.advance(ws[0].n_steps)
                n = noise[0]
                out.append(sim.read_iq(0) if n is None else sim.read_iq(0, n[0], n[1], n[2]))
            finally:
                sim.close()
            continue
        b = Batch([run_config(w) for w in ws], [s.ptr if s else None for s in setups])
        try:
            b.advance(max(w.n_steps for w in ws))
            for q, n in enumerate(noise):
                out.append(b.read_iq(q, 0) if n is None else b.read_iq(q, 0, n[0], n[1], n[2]))
        finally:
            b.close()
    return out


def write_examples(cfg, indices, out_dir: str | os.PathLike | None = None) -> list:
    """run_examples, each result written as <out_dir>/example_%06d.iq in
    rfsyn's .iq format (job.output_dir when out_dir is None)."""
    from . import iq_write

    out_dir = out_dir if out_dir is not None else (get(cfg, "job", "output_dir") or PRESET[("job", "output_dir")])
    os.makedirs(out_dir, exist_ok=True)
    paths = []
    for i, iq in zip(indices, run_examples(cfg, indices)):
        p = os.path.join(out_dir, f"example_{i:06d}.iq")
        iq_write(p, iq)
        paths.append(p)
    return paths
