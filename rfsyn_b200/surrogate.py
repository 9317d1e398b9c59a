"""Transfer-function surrogate: a small MLP ensemble that maps a scene's
parameter vector to its complex tx -> rx transfer function, trained on
data the batched FDTD generates, with plain FDTD as the fallback whenever
the ensemble disagrees.  rfsyn has no learned component.

Scene vector (54 values): 8 scatterers x 6 values, zero-padded, then the
tx position and the rx - tx vector, all scaled to O(1).  Each scatterer is
described relative to the tx / rx pair -- its distances to both, its excess
path length over the direct path, its radius, eps_r and log10 sigma -- and
the scatterers are sorted by excess path length, so that the network sees a
canonical order (the field at the receiver does not depend on the order in
which scatterers are listed).
Output (512 values): the de-embedded transfer function
    G(f) = H(f) / Ez_free(f; d, theta)
at 256 bins, real parts then imaginary parts, divided by one scale learned
from the training set.  H(f) = P(f) / S(f): the receive probe's spectrum
over the spectrum of the transmitted waveform, both with the engine's DFT
convention.  Ez_free is the z component of the free-space field of a
z-directed elementary dipole at the receiver (distance d, polar angle
theta from the dipole axis), near, intermediate and far terms:
    E_r     = cos(theta) / (2 pi d^2) (1 + 1/(jkd)) e^{-jkd}
    E_theta = j k sin(theta) / (4 pi d) (1 + 1/(jkd) - 1/(kd)^2) e^{-jkd}
    Ez      = E_r cos(theta) - E_theta sin(theta)
(constant factors dropped; the soft source is a current element whose
moment is proportional to the injected value).  Dividing it out removes the
spreading, delay and near-field structure of the direct path, so the
network learns what the scatterers and the grid add to it.

The network (forward, backward, Adam) runs on the GPU through
fdtd_b200_mlp_* (rfsyn_b200/csrc/mlp.cu); every FDTD run goes through the
batch engine (fdtd_b200_batch_*).
"""
from __future__ import annotations

import functools
import math
import time
from dataclasses import dataclass

import numpy as np

from . import C0, FIELD_EZ, FP32, WAVE_MOD_GAUSSIAN, Batch, Mlp
from . import ranks as rk
from . import scenes as sc

N_SCAT = 8
N_FEAT = 6 * N_SCAT + 6
N_BINS = 256


def c5_scenes(seed: int, n_scenes: int, n: int = 48, n_steps: int = 1500, npml: int = 8, max_scat: int = N_SCAT,
              precision: int = FP32) -> list[sc.Workload]:
    """Surrogate scenes: n^3 cells at dx 2 mm, npml-cell CPML; 0..max_scat
    dielectric spheres (radius U[2,8] cells, eps_r U[1,10], sigma
    log-U[1e-4,1] S/m) clear of the CPML; one soft Ez transmitter
    (Gaussian-modulated sinusoid f0 6 GHz, tau = 2/(pi 8 GHz), t0 = 4 tau)
    and 4 Ez receivers at interior positions at least 4 cells from it;
    256 DFT bins linear over 1..11 GHz.  Scene s draws from PCG32(seed, s)."""
    tau = 2.0 / (math.pi * 8e9)
    freqs = list(np.linspace(1e9, 11e9, N_BINS))
    lo, hi = npml + 3, n - npml - 3
    out = []
    for s in range(n_scenes):
        rng = sc.Pcg32(seed, s)
        spheres = []
        for _ in range(rng.randint(0, max_scat + 1)):
            r = rng.range(2.0, min(8.0, (n - 2 * npml - 6) / 2.0))
            c = [rng.range(npml + r + 2, n - npml - r - 2) for _ in range(3)]
            spheres.append((c[0], c[1], c[2], r, rng.range(1.0, 10.0), rng.log_range(1e-4, 1.0), None))
        tx = [rng.randint(lo, hi) for _ in range(3)]
        rxs = []
        while len(rxs) < 4:
            p = [rng.randint(lo, hi) for _ in range(3)]
            if sum((a - b) ** 2 for a, b in zip(p, tx)) >= 16:
                rxs.append(p)
        out.append(sc.Workload(
            name=f"c5_scene{s}", nx=n, ny=n, nz=n, dx=2e-3, n_steps=n_steps, npml=npml, precision=precision,
            sources=[dict(i=tx[0], j=tx[1], k=tx[2], component=FIELD_EZ, mode=0, amplitude=1.0,
                          waveform=WAVE_MOD_GAUSSIAN, p0=6e9, p1=4.0 * tau, p2=tau)],
            probes=[dict(i=p[0], j=p[1], k=p[2], component=FIELD_EZ) for p in rxs], freqs=freqs, spheres=spheres))
    return out


def features(w: sc.Workload, rx: int) -> np.ndarray:
    """The 54-value scene vector of receiver rx."""
    n = float(w.nx)
    f = np.zeros(N_FEAT, dtype=np.float64)
    s, p = w.sources[0], w.probes[rx]
    tx = np.array([s["i"], s["j"], s["k"]], dtype=np.float64)
    rv = np.array([p["i"], p["j"], p["k"]], dtype=np.float64)
    direct = float(np.linalg.norm(rv - tx))
    rows = []
    for (cx, cy, cz, r, eps, sig, _) in w.spheres[:N_SCAT]:
        c = np.array([cx, cy, cz])
        dt_, dr_ = float(np.linalg.norm(c - tx)), float(np.linalg.norm(c - rv))
        excess = dt_ + dr_ - direct
        rows.append((excess, (dt_ / n, dr_ / n, excess / n, r / n, (eps - 1.0) / 9.0,
                              (math.log10(sig) + 4.0) / 4.0)))
    rows.sort(key=lambda t: t[0])
    for q, (_, v) in enumerate(rows):
        f[6 * q: 6 * q + 6] = v
    f[48:51] = tx / n
    f[51:54] = (rv - tx) / n
    return f


def source_spectrum(w: sc.Workload) -> np.ndarray:
    """DFT of the transmitted waveform samples (engine convention: sample n
    at t = n dt for the source, weight dt).  Scenes that share the waveform,
    dt, step count and bins share one (read-only) array: the transform
    costs ~10-20 ms of host time and every surrogate scene has the same."""
    s = w.sources[0]
    return _source_spectrum(float(s["amplitude"]), float(s["p0"]), float(s["p1"]), float(s["p2"]), float(w.dt),
                            int(w.n_steps), tuple(float(f) for f in w.freqs))


@functools.lru_cache(maxsize=16)
def _source_spectrum(amplitude: float, p0: float, p1: float, p2: float, dt: float, n_steps: int,
                     freqs: tuple) -> np.ndarray:
    t = np.arange(n_steps) * dt
    u = (t - p1) / p2
    v = amplitude * np.exp(-u * u) * np.sin(2.0 * math.pi * p0 * (t - p1))
    f = np.asarray(freqs)
    S = (v[None, :] * np.exp(-2j * math.pi * f[:, None] * t[None, :])).sum(axis=1) * dt
    S.setflags(write=False)
    return S


def ez_free(w: sc.Workload, rx: int) -> np.ndarray:
    """Ez of a z-directed elementary dipole at the transmitter, observed at
    receiver rx, over the scene's bins (constant factors dropped)."""
    s, p = w.sources[0], w.probes[rx]
    v = np.asarray([(p[a] - s[a]) * w.dx for a in "ijk"], dtype=np.float64)
    d = float(np.linalg.norm(v))
    ct = v[2] / d
    st = math.sqrt(max(0.0, 1.0 - ct * ct))
    k = 2.0 * math.pi * np.asarray(w.freqs) / C0
    kd = k * d
    ph = np.exp(-1j * kd)
    er = ct / (2.0 * math.pi * d * d) * (1.0 + 1.0 / (1j * kd)) * ph
    eth = 1j * k * st / (4.0 * math.pi * d) * (1.0 + 1.0 / (1j * kd) - 1.0 / (kd * kd)) * ph
    return er * ct - eth * st


def _deembed(w: sc.Workload, rx: int) -> np.ndarray:
    return 1.0 / ez_free(w, rx)


def transfer_functions(ws: list[sc.Workload], chunk: int = 512, timings: dict | None = None):
    """Runs the scenes with the batch engine; returns the scene vectors
    [4 n, 54] and transfer functions H [4 n, 256] (complex)."""
    X, H = [], []
    run_ms = 0.0
    for c0 in range(0, len(ws), chunk):
        part = ws[c0:c0 + chunk]
        setups = [sc.scene_setup(w) for w in part]
        b = Batch([sc.run_config(w) for w in part], [st.ptr if st else None for st in setups])
        run_ms += b.advance_timed(part[0].n_steps)
        for q, w in enumerate(part):
            S = source_spectrum(w)
            dft = b.dft(q)
            for rx in range(len(w.probes)):
                X.append(features(w, rx))
                H.append(dft[rx] / S)
        b.close()
    if timings is not None:
        timings["fdtd_ms"] = timings.get("fdtd_ms", 0.0) + run_ms
    return np.asarray(X), np.asarray(H)


def sharded_transfer_functions(ws: list[sc.Workload], r: rk.Ranks, device: str = "cuda", timings: dict | None = None,
                               tf=transfer_functions):
    """transfer_functions over several ranks: rank r runs its contiguous
    shard of the scenes, then every rank receives all rows in scene order."""
    mine = [ws[q] for q in rk.shard(len(ws), r)]
    X, H = tf(mine, timings=timings) if mine else (np.zeros((0, N_FEAT)), np.zeros((0, N_BINS), complex))
    return rk.gather_rows(r, np.asarray(X, dtype=np.float64), device), \
        rk.gather_rows(r, np.asarray(H, dtype=np.complex128), device)


def scene_transfer_targets(ws: list[sc.Workload], H: np.ndarray) -> np.ndarray:
    """G = H * deembed for every (scene, receiver) row of H (complex)."""
    D = np.asarray([_deembed(w, rx) for w in ws for rx in range(len(w.probes))])
    return H * D


def rel_err(pred: np.ndarray, true: np.ndarray) -> np.ndarray:
    """Per-row relative L2 error over the frequency bins."""
    return np.linalg.norm(pred - true, axis=-1) / np.maximum(np.linalg.norm(true, axis=-1), 1e-300)


@dataclass
class Prediction:
    H: np.ndarray          # predicted transfer functions (rows x 256)
    spread: np.ndarray     # ensemble disagreement per row (relative)


class Surrogate:
    """An ensemble of GPU MLPs over the de-embedded transfer function.  With
    several ranks each rank holds, trains and evaluates its share of the
    members (ranks.members_of); predictions are gathered on every rank."""

    def __init__(self, members: int = 5, width: int = 512, depth: int = 4, seed: int = 0,
                 r: rk.Ranks | None = None, device: str = "cuda"):
        self.r = r or rk.Ranks(0, 1, 0)
        self.device = device
        self.members = rk.members_of(members, self.r)
        self.nets = [Mlp(N_FEAT, width, depth, 2 * N_BINS, seed=seed + 7919 * q) for q in self.members]
        self.scale = 1.0
        self.seed = seed

    def _enc(self, G: np.ndarray) -> np.ndarray:
        return np.concatenate([G.real, G.imag], axis=1) / self.scale

    def _dec(self, Y: np.ndarray) -> np.ndarray:
        return (Y[:, :N_BINS] + 1j * Y[:, N_BINS:]) * self.scale

    def fit(self, X: np.ndarray, G: np.ndarray, steps: int = 20000, batch: int = 256, lr: float = 1e-3) -> list:
        """Trains every member on (X, G); returns the final batch losses."""
        self.scale = float(np.sqrt(np.mean(np.abs(G) ** 2)))
        T = self._enc(G).astype(np.float32)
        losses = []
        for q, net in zip(self.members, self.nets):
            net.set_data(X.astype(np.float32), T)
            losses.append(net.train(steps, batch=batch, lr=lr, seed=self.seed + 104729 * q + 1))
        return list(rk.gather_rows(self.r, np.asarray(losses, dtype=np.float64), self.device))

    def predict_g(self, X: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        local = np.stack([self._dec(net.predict(X.astype(np.float32)).astype(np.float64)) for net in self.nets]) \
            if self.nets else np.zeros((0, len(X), N_BINS), complex)
        outs = rk.gather_rows(self.r, local, self.device)
        mean = outs.mean(axis=0)
        spread = np.sqrt(np.mean(np.sum(np.abs(outs - mean) ** 2, axis=-1), axis=0)) / np.maximum(
            np.linalg.norm(mean, axis=-1), 1e-300)
        return mean, spread

    def predict(self, ws: list[sc.Workload], X: np.ndarray | None = None) -> Prediction:
        if X is None:
            X = np.asarray([features(w, rx) for w in ws for rx in range(len(w.probes))])
        G, spread = self.predict_g(X)
        D = np.asarray([_deembed(w, rx) for w in ws for rx in range(len(w.probes))])
        return Prediction(H=G / D, spread=spread)

    def close(self):
        for n in self.nets:
            n.close()


def infer_with_fallback(sur: Surrogate, ws: list[sc.Workload], threshold: float = 0.02) -> dict:
    """Transfer functions of every (scene, receiver): the ensemble mean where
    the ensemble agrees (spread <= threshold for all the scene's receivers),
    the batched FDTD otherwise (the fallback scenes sharded over the ranks).
    Returns H, which scenes fell back and the wall time of each part."""
    t0 = time.perf_counter()
    pred = sur.predict(ws)
    t_sur = time.perf_counter() - t0
    nrx = [len(w.probes) for w in ws]
    rows = np.cumsum([0] + nrx)
    fall = [q for q in range(len(ws)) if np.any(pred.spread[rows[q]:rows[q + 1]] > threshold)]
    H = pred.H.copy()
    t1 = time.perf_counter()
    timings: dict = {}
    if fall:
        _, Hf = sharded_transfer_functions([ws[q] for q in fall], sur.r, sur.device, timings=timings)
        r = 0
        for q in fall:
            H[rows[q]:rows[q + 1]] = Hf[r:r + nrx[q]]
            r += nrx[q]
    t_fdtd = time.perf_counter() - t1
    return {"H": H, "fallback": fall, "spread": pred.spread, "surrogate_s": t_sur, "fdtd_s": t_fdtd,
            "fdtd_device_ms": timings.get("fdtd_ms", 0.0)}
