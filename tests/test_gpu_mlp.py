"""Surrogate network kernels against the CPU reference (oracle/mlp_oracle.py):
FP32 forward and gradient (relative 1e-4), BF16 tensor-core inference against
the FP32 forward (2e-2 of the output scale), and training that lowers the loss."""
import numpy as np
import pytest

import openrcwa_b200 as o
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def test_forward_and_gradient_match_cpu(eng):
    rng = np.random.default_rng(0)
    net = o.Mlp(eng, 11, 64, 3, 52, seed=3)
    X = rng.uniform(-1, 1, (96, 11)).astype(np.float32)
    Y = rng.uniform(0, 1, (96, 52)).astype(np.float32)
    p = net.get_params()
    P = net.predict(X, tensor_cores=False)
    Pref, _, _ = mo.forward(p, net.dims, X)
    assert np.max(np.abs(P - Pref)) < 1e-4 * max(1.0, np.max(np.abs(Pref)))
    loss, g = net.loss_grad(X, Y)
    lref, gref = mo.loss_grad(p, net.dims, X, Y)
    assert abs(loss - lref) < 1e-5 * max(1.0, lref)
    assert np.max(np.abs(g - gref)) < 1e-4 * np.max(np.abs(gref))
    net.close()


@pytest.mark.parametrize("rows", [1, 127, 128, 1000, 65536])
def test_tensor_core_inference(eng, rows):
    rng = np.random.default_rng(rows)
    net = o.Mlp(eng, 11, 256, 4, 52, seed=7)
    X = rng.uniform(-1, 1, (rows, 11)).astype(np.float32)
    Ptc = net.predict(X, tensor_cores=True)
    P32 = net.predict(X, tensor_cores=False)
    scale = max(1.0, float(np.max(np.abs(P32))))
    assert np.all(np.isfinite(Ptc))
    assert np.max(np.abs(Ptc - P32)) < 2e-2 * scale
    net.close()


def test_training_lowers_loss(eng):
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (4096, 11)).astype(np.float32)
    Y = np.stack([np.sin(2 * X[:, 0]) * X[:, 1], np.cos(X[:, 2] + X[:, 3]), X[:, 4] ** 2], axis=1).astype(np.float32)
    net = o.Mlp(eng, 11, 128, 3, 3, seed=1)
    net.set_data(X, Y)
    loss = net.train(epochs=30, batch=256, lr=2e-3, seed=2)
    assert loss[-1] < 0.05 * loss[0]
    P = net.predict(X[:512], tensor_cores=True)
    assert np.sqrt(np.mean((P - Y[:512]) ** 2)) < 0.05
    net.close()
