"""The VCA surrogate network on the GPU (BF16 tensor-core products, FP32
accumulation, Adam) against its CPU restatement oracle/mlp_port.py: forward
pass and gradients at the same rounding points, then training."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def port():
    from oracle import mlp_port
    return mlp_port


def _net(width=64, seed=3):
    from pyqcm_b200 import surrogate as S
    return S.MLP(n_in=4, width=width, seed=seed)


def test_forward_matches_port(port):
    net = _net()
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (100, 4)).astype(np.float32)
    y = net(x)
    want, _ = port.forward(net.blocks(), x, 4)
    # BF16 activations: a rounding that lands differently moves an output by ~2^-9 of a term
    assert np.max(np.abs(y - want)) < 2e-3 * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("width", [64, 256])
def test_gradients_match_port(port, width):
    net = _net(width=width, seed=11)
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (128, 4)).astype(np.float32)
    t = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2]).astype(np.float32)
    g, loss = net.gradients(x, t)
    loss_ref, g_ref = port.gradients(net.blocks(), x, t, 4)
    assert abs(loss - loss_ref) < 1e-3 * max(1.0, loss_ref)
    for i, (a, b) in enumerate(zip(net.blocks(g), g_ref)):
        b = np.asarray(b).reshape(np.shape(a)) if np.ndim(a) else b
        err = np.linalg.norm(np.asarray(a, dtype=np.float64) - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 2e-2, (i, err)


def test_training_fits_a_smooth_function():
    net = _net(width=256, seed=5)
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (2048, 4)).astype(np.float32)
    f = lambda x: (0.5 * x[:, 0] ** 2 - 0.3 * x[:, 1] * x[:, 2] + 0.2 * np.cos(2 * x[:, 3])).astype(np.float32)
    losses = net.train(x, f(x), epochs=300, batch=256, lr=1e-3, seed=0)
    xt = rng.uniform(-1, 1, (512, 4)).astype(np.float32)
    rmse = np.sqrt(np.mean((net(xt) - f(xt)) ** 2))
    assert losses[-1] < 0.01 * losses[0]
    assert rmse < 0.02, rmse
