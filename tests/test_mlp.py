"""The surrogate network's GPU kernels (BF16 tensor-core GEMMs with FP32
accumulation, GELU epilogues, MSE gradient, Adam) against the CPU oracle
(oracle/mlp_oracle.py, FP64 with the pipeline's bfloat16 rounding points).
The products run on mma.sync tiles; with RFSYN_FDTD_MLP_GEMM=tcgen05,
those whose rows are a multiple of 128 run on the tcgen05 tensor cores
(accumulators in tensor memory): batches of 128 and 256 put every product
there, checked against the oracle and against the mma.sync products of the
same network.

Tolerances: the GPU and the oracle round the same operands to bfloat16, so
they differ by FP32 accumulation order and by an occasional operand that
lands on the other side of a bfloat16 rounding boundary: 2e-3 relative L2
on gradients and outputs, 1e-4 on the loss."""
from __future__ import annotations

import numpy as np
import pytest

import rfsyn_b200 as rb
from oracle.mlp_oracle import MlpOracle

pytestmark = pytest.mark.gpu
SHAPE = dict(n_in=54, width=128, depth=2, n_out=128)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def data():
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (128, SHAPE["n_in"]))
    Y = rng.normal(0, 1, (128, SHAPE["n_out"]))
    return X, Y


def test_gradient_matches_oracle(data):
    X, Y = data
    net = rb.Mlp(**SHAPE, seed=3)
    orc = MlpOracle(**SHAPE)
    p = net.params().astype(np.float64)
    assert p.size == orc.n_params
    loss, g = net.grad(X[:64], Y[:64])
    loss_o, g_o = orc.loss_grad(p, X[:64], Y[:64], bf16=True)
    assert abs(loss - loss_o) <= 1e-4 * abs(loss_o)
    assert _rel(g.astype(np.float64), g_o) < 2e-3
    # per layer as well (the first layer's gradient has passed every GELU')
    o = 0
    for i, n in orc.shapes:
        k = n * i + n
        assert _rel(g[o:o + k].astype(np.float64), g_o[o:o + k]) < 2e-3
        o += k
    net.close()


def test_forward_matches_oracle(data):
    X, _ = data
    net = rb.Mlp(**SHAPE, seed=4)
    orc = MlpOracle(**SHAPE)
    p = net.params().astype(np.float64)
    out = net.predict(X[:100])           # 100 rows: a padded last batch
    want = orc.predict(p, X[:100], bf16=True)
    assert out.shape == want.shape
    assert _rel(out.astype(np.float64), want) < 2e-3
    net.close()


def test_adam_step_matches_oracle(data):
    """One training step on a one-batch data set: the GPU's Adam update
    (learning rate 1e-3 at step 0 of 10) equals the oracle's applied to the
    oracle gradient, element by element within the bfloat16 rounding."""
    X, Y = data
    net = rb.Mlp(**SHAPE, seed=6)
    orc = MlpOracle(**SHAPE)
    p0 = net.params().astype(np.float64)
    net.set_data(X[:64], Y[:64])
    net.train(1, batch=64, lr=1e-3, seed=1)
    p1 = net.params().astype(np.float64)
    _, g = orc.loss_grad(p0, X[:64], Y[:64], bf16=True)
    m = np.zeros_like(p0)
    want, _, _ = orc.adam(p0, g, m, m.copy(), 0, 1e-3, 1)
    d_gpu, d_want = p1 - p0, want - p0
    # the first Adam step moves every weight by lr * g / (|g| + eps): sign
    # agreement wherever the gradient is not negligible
    big = np.abs(g) > 1e-3 * np.abs(g).max()
    agree = np.abs(d_gpu[big] - d_want[big]) <= 1e-6 + 1e-3 * np.abs(d_want[big])
    assert agree.mean() > 0.999, agree.mean()
    net.close()


def test_training_reduces_loss():
    rng = np.random.default_rng(8)
    X = rng.uniform(-1, 1, (2048, SHAPE["n_in"]))
    W = rng.normal(0, 1, (SHAPE["n_in"], SHAPE["n_out"])) / np.sqrt(SHAPE["n_in"])
    Y = np.sin(X @ W)
    net = rb.Mlp(**SHAPE, seed=9)
    loss0, _ = net.grad(X[:256], Y[:256])
    net.set_data(X, Y)
    loss = net.train(1500, batch=256, lr=2e-3, seed=2)
    assert loss < 0.1 * loss0, (loss0, loss)
    err = np.mean((net.predict(X[:512]) - Y[:512]) ** 2)
    assert err < 0.1 * loss0
    net.close()


@pytest.fixture(scope="module")
def data256():
    rng = np.random.default_rng(15)
    X = rng.uniform(-1, 1, (256, SHAPE["n_in"]))
    Y = rng.normal(0, 1, (256, SHAPE["n_out"]))
    return X, Y


@pytest.mark.parametrize("batch", [128, 256])
def test_tensor_core_gradient_matches_oracle(data256, batch, monkeypatch):
    X, Y = data256
    monkeypatch.setenv("RFSYN_FDTD_MLP_GEMM", "tcgen05")
    net = rb.Mlp(**SHAPE, seed=11)
    orc = MlpOracle(**SHAPE)
    p = net.params().astype(np.float64)
    n0 = net.tensor_core_launches()
    loss, g = net.grad(X[:batch], Y[:batch])
    # every product of the pass (forward, dW, dX) ran on the tcgen05 path
    assert net.tensor_core_launches() - n0 == 3 * (SHAPE["depth"] + 1) - 1
    loss_o, g_o = orc.loss_grad(p, X[:batch], Y[:batch], bf16=True)
    assert abs(loss - loss_o) <= 1e-4 * abs(loss_o)
    assert _rel(g.astype(np.float64), g_o) < 2e-3
    out = net.predict(X[:batch])
    assert _rel(out.astype(np.float64), orc.predict(p, X[:batch], bf16=True)) < 2e-3
    net.close()


def test_tensor_core_products_agree_with_mma_sync(data256, monkeypatch):
    """The same network, batch and data through both product kernels: they
    differ only by the FP32 accumulation order."""
    X, Y = data256
    monkeypatch.setenv("RFSYN_FDTD_MLP_GEMM", "tcgen05")
    a = rb.Mlp(**SHAPE, seed=12)
    monkeypatch.delenv("RFSYN_FDTD_MLP_GEMM")
    b = rb.Mlp(**SHAPE, seed=12)
    la, ga = a.grad(X, Y)
    lb, gb = b.grad(X, Y)
    assert a.tensor_core_launches() > 0 and b.tensor_core_launches() == 0
    assert abs(la - lb) <= 1e-5 * abs(lb)
    assert _rel(ga.astype(np.float64), gb.astype(np.float64)) < 1e-3
    a.close()
    b.close()

