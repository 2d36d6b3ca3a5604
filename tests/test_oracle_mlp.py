"""The MLP oracle (oracle/mlp_oracle.py) against central finite differences, in FP64."""
import numpy as np

import mlp_oracle as M


def test_gelu_derivative_matches_finite_differences():
    x = np.linspace(-6.0, 6.0, 97)
    h = 1e-6
    fd = (M.gelu(x + h) - M.gelu(x - h)) / (2 * h)
    np.testing.assert_allclose(M.gelu_grad(x), fd, rtol=0, atol=1e-8)
    # known values: GELU(0) = 0, GELU(x) -> x for large x, -> 0 for very negative x
    assert M.gelu(0.0) == 0.0
    np.testing.assert_allclose(M.gelu(np.array([8.0, -8.0])), [8.0, 0.0], atol=1e-12)


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    I, H, O, B = 4, 7, 5, 6
    n = H * I + H + H * H + H + O * H + O
    p = rng.normal(size=n) * 0.5
    x = rng.normal(size=(B, I))
    t = rng.normal(size=(B, O))
    loss, g = M.loss_gradient(p, x, t, I, H, O)
    h = 1e-6
    fd = np.zeros(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = h
        fd[i] = (M.loss_gradient(p + e, x, t, I, H, O)[0] - M.loss_gradient(p - e, x, t, I, H, O)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-9)
    y, _ = M.forward(p, x, I, H, O)
    assert abs(loss - 0.5 * np.sum((y - t) ** 2) / B) < 1e-14
