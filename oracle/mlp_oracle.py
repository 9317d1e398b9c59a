"""TEST INFRASTRUCTURE -- CPU restatement of the surrogate network.

FP64 NumPy forward pass, mean-squared-error gradient and Adam update of the
multilayer perceptron that rfsyn_b200/csrc/mlp.cu trains on the GPU (rfsyn
has no learned component, so nothing in rfsyn pins it; the gradient is
pinned here by central finite differences, see tests/test_mlp_oracle.py).

Layers: n_in (zero-padded to kin) -> width (GELU) -> ... -> n_out; GELU is
the exact 0.5 x (1 + erf(x / sqrt 2)).  Parameters are flat, layer by layer:
W (out x in, row-major) then b, as fdtd_b200_mlp_get_params.

With bf16=True the BF16 rounding points of the GPU pipeline are applied
(inputs, weights and the activations / gradients fed to the tensor-core
GEMMs are rounded to bfloat16, round-to-nearest-even); accumulation stays
FP64, so the GPU result differs from it only by FP32 summation.
Only tests may import this module.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf

SQRT1_2 = 1.0 / math.sqrt(2.0)


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x * SQRT1_2))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x * SQRT1_2)) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


class MlpOracle:
    def __init__(self, n_in: int, width: int, depth: int, n_out: int):
        self.n_in, self.width, self.depth, self.n_out = n_in, width, depth, n_out
        self.kin = (n_in + 63) // 64 * 64
        self.shapes = [(width if l else self.kin, width) for l in range(depth)] + [(width, n_out)]

    @property
    def n_params(self) -> int:
        return sum(i * o + o for i, o in self.shapes)

    def unpack(self, p: np.ndarray):
        out, o = [], 0
        for i, n in self.shapes:
            W = p[o:o + n * i].reshape(n, i)
            o += n * i
            b = p[o:o + n]
            o += n
            out.append((W.astype(np.float64), b.astype(np.float64)))
        return out

    def pad(self, X: np.ndarray) -> np.ndarray:
        Xp = np.zeros((X.shape[0], self.kin))
        Xp[:, : self.n_in] = X
        return Xp

    def forward(self, p: np.ndarray, X: np.ndarray, bf16: bool = False):
        r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
        layers = self.unpack(p)
        a = r(self.pad(X))
        acts, pres = [a], []
        for l, (W, b) in enumerate(layers):
            z = a @ r(W).T + b
            if l < len(layers) - 1:
                pres.append(z)
                a = r(gelu(z))
                acts.append(a)
            else:
                out = z
        return out, acts, pres

    def predict(self, p, X, bf16=False):
        return self.forward(p, X, bf16)[0]

    def loss_grad(self, p: np.ndarray, X: np.ndarray, Y: np.ndarray, bf16: bool = False):
        """Mean squared error over all outputs and its gradient (flat)."""
        r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
        layers = self.unpack(p)
        out, acts, pres = self.forward(p, X, bf16)
        M, N = out.shape
        e = out - Y
        loss = float(np.sum(e * e) / (M * N))
        d = 2.0 * e / (M * N)          # FP32 in the pipeline
        grads = [None] * len(layers)
        for l in range(len(layers) - 1, -1, -1):
            W, b = layers[l]
            gW = r(d).T @ acts[l]
            gb = d.sum(axis=0)
            grads[l] = (gW, gb)
            if l > 0:
                d = (r(d) @ r(W)) * gelu_grad(pres[l - 1])
        flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
        return loss, flat

    @staticmethod
    def adam(p, g, m, v, step, lr0, total_steps, beta1=0.9, beta2=0.999, eps=1e-8):
        """One Adam update (step = updates done before this one), learning
        rate lr0 * 0.5 (1 + cos(pi step / total_steps)); returns p, m, v."""
        s = step + 1
        frac = min(1.0, step / max(1, total_steps))
        lr = lr0 * 0.5 * (1.0 + math.cos(math.pi * frac))
        m = beta1 * m + (1 - beta1) * g
        v = beta2 * v + (1 - beta2) * g * g
        mh = m / (1 - beta1 ** s)
        vh = v / (1 - beta2 ** s)
        return p - lr * mh / (np.sqrt(vh) + eps), m, v
