"""CPU oracle of the learned warm start's network (TEST INFRASTRUCTURE ONLY).

FP64 numpy restatement of the MLP that libfemmgpu trains and evaluates on the GPU
(femm-gpu_b200/csrc/mlp.cu): inputs -> hidden -> hidden -> outputs, exact-erf GELU after
each hidden layer, loss 0.5 / batch * sum (y - t)^2, parameter vector
[W1 (H x I), b1 (H), W2 (H x H), b2 (H), W3 (O x H), b3 (O)].  The network has no
counterpart in the reference; this oracle is pinned by central finite differences in the
CPU tests and checks the GPU gradients in the GPU tests.
"""
import numpy as np
from scipy.special import erf

SQRT_HALF = np.sqrt(0.5)
INV_SQRT_2PI = 1.0 / np.sqrt(2.0 * np.pi)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x * SQRT_HALF))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x * SQRT_HALF)) + x * INV_SQRT_2PI * np.exp(-0.5 * x * x)


def split(p, I, H, O):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((H, I), (H,), (H, H), (H,), (O, H), (O,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == p.size
    return out


def forward(p, x, I, H, O):
    W1, b1, W2, b2, W3, b3 = split(p, I, H, O)
    x = np.asarray(x, np.float64)
    h1 = x @ W1.T + b1
    a1 = gelu(h1)
    h2 = a1 @ W2.T + b2
    a2 = gelu(h2)
    y = a2 @ W3.T + b3
    return y, (x, h1, a1, h2, a2)


def loss_gradient(p, x, t, I, H, O):
    W1, b1, W2, b2, W3, b3 = split(p, I, H, O)
    y, (x, h1, a1, h2, a2) = forward(p, x, I, H, O)
    B = x.shape[0]
    e = y - np.asarray(t, np.float64)
    loss = 0.5 * np.sum(e * e) / B
    dy = e / B
    gW3 = dy.T @ a2
    gb3 = dy.sum(axis=0)
    d2 = (dy @ W3) * gelu_grad(h2)
    gW2 = d2.T @ a1
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * gelu_grad(h1)
    gW1 = d1.T @ x
    gb1 = d1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
