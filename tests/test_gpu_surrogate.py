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


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (100, 16, 16), (300, 256, 272), (256, 48, 4096), (16, 144, 80)])
def test_tensor_product_matches_exact_products(M, N, K):
    """The tcgen05 product on shapes with partial tiles (M not a multiple of 128,
    N not a multiple of the 128-column tile, K not a multiple of the 64-element
    round) against the exact products of the same BF16 inputs summed in float64.
    Products of two BF16 numbers are exact in FP32, so the only difference is the
    FP32 accumulation: bounded by K * 2^-24 * sum |a b| per entry."""
    from pyqcm_b200 import surrogate as S
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    a = S.to_bf16_bits(rng.standard_normal((M, K)).astype(np.float32))
    b = S.to_bf16_bits(rng.standard_normal((N, K)).astype(np.float32))
    c = S.tensor_product(a, b)
    A = S.from_bf16_bits(a).astype(np.float64)
    B = S.from_bf16_bits(b).astype(np.float64)
    want = A @ B.T
    bound = K * 2.0 ** -23 * (np.abs(A) @ np.abs(B).T) + 1e-30
    assert np.all(np.abs(c - want) <= bound), float(np.max(np.abs(c - want) / bound))
