"""The oracle's restatement of the learned-smoother network: its analytic
gradient against central finite differences, and the BF16 rounding rule."""
import numpy as np

from oracle.binding import mlp_forward, mlp_loss_grad

NP = 4995


def _params(seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, 0.3, NP)
    return p


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _params()
    x = rng.normal(size=(37, 9))
    t = rng.normal(size=(37, 3))
    loss, g = mlp_loss_grad(p, x, t, bf16=False)
    assert loss > 0
    idx = rng.choice(NP, 60, replace=False)
    idx = np.concatenate([idx, [0, 575, 576, 639, 640, 4735, 4736, 4799, 4800, 4991, 4992, 4994]])
    h = 1e-6
    for q in idx:
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (mlp_loss_grad(pp, x, t, bf16=False)[0] - mlp_loss_grad(pm, x, t, bf16=False)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 + 1e-5 * abs(fd), (q, fd, g[q])


def test_oracle_bf16_forward_rounds_like_the_tensor_cores():
    rng = np.random.default_rng(2)
    p = _params(3)
    x = rng.normal(size=(50, 9))
    y64 = mlp_forward(p, x, bf16=False)
    y16 = mlp_forward(p, x, bf16=True)
    rel = np.abs(y16 - y64).max() / np.abs(y64).max()
    assert 1e-4 < rel < 5e-2          # BF16 keeps 8 significant bits
    # a value exactly representable in BF16 passes through unchanged
    p2 = np.zeros(NP)
    p2[4992] = 1.5                    # b3[0]
    assert mlp_forward(p2, np.zeros((1, 9)), bf16=True)[0, 0] == 1.5
