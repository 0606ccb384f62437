"""The learned smoother's network on the GPU: tcgen05 tensor-core forward and
the hand-written backward against the FP64 oracle with the same BF16
roundings, and a training run through the library's own trainer."""
import numpy as np
import pytest

from multigridsoftbody_b200.learned import MLP, NUM_PARAMS
from oracle.binding import mlp_forward, mlp_loss_grad

pytestmark = pytest.mark.gpu


def test_forward_matches_oracle(lib, oracle_built):
    net = MLP(seed=5)
    rng = np.random.default_rng(0)
    p = net.params.astype(np.float64)
    for n in (1, 127, 128, 1000, 40000):
        x = rng.normal(size=(n, 9)).astype(np.float32)
        y = net.forward(x)
        want = mlp_forward(p, x.astype(np.float64), bf16=True)
        scale = np.abs(want).max()
        # FP32 accumulation order and BF16 rounding-boundary flips of hidden
        # activations are the only differences
        assert np.abs(y - want).max() <= 2e-2 * scale, (n, np.abs(y - want).max(), scale)
        assert np.abs(y - want).mean() <= 2e-3 * scale
    net.close()


def test_gradient_matches_oracle(lib, oracle_built):
    net = MLP(seed=7)
    rng = np.random.default_rng(1)
    x = rng.normal(size=(300, 9)).astype(np.float32)
    t = rng.normal(size=(300, 3)).astype(np.float32)
    loss, g = net.loss_grad(x, t)
    lo, go = mlp_loss_grad(net.params.astype(np.float64), x.astype(np.float64), t.astype(np.float64), bf16=True)
    assert abs(loss - lo) <= 1e-4 * lo
    assert np.linalg.norm(g - go) <= 1e-3 * np.linalg.norm(go)
    # per block of parameters
    for a, b in ((0, 576), (576, 640), (640, 4736), (4736, 4800), (4800, 4992), (4992, 4995)):
        assert np.linalg.norm(g[a:b] - go[a:b]) <= 3e-3 * np.linalg.norm(go[a:b]) + 1e-7, (a, b)
    net.close()


def test_training_fits_a_linear_map(lib):
    """A 3x9 linear map is learnt to a small fraction of its variance."""
    rng = np.random.default_rng(2)
    A = rng.normal(size=(3, 9)).astype(np.float32) * 0.5
    x = rng.normal(size=(20000, 9)).astype(np.float32)
    t = x @ A.T
    net = MLP(seed=3)
    losses = net.train(x, t, steps=1500, batch=2048, lr=3e-3, seed=9)
    assert np.isfinite(losses).all()
    assert losses[-50:].mean() < 0.02 * losses[:10].mean(), (losses[:10].mean(), losses[-50:].mean())
    y = net.forward(x[:1000])
    assert np.mean((y - t[:1000]) ** 2) < 0.02 * np.mean(t[:1000] ** 2)
    p = net.params
    assert p.shape == (NUM_PARAMS,) and np.isfinite(p).all()
    net.close()
