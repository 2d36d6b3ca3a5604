"""GPU tests of the learned warm start: the network's kernels against the FP64 CPU oracle
(oracle/mlp_oracle.py), the reduced basis, the residual guard, and what the trained
network gains over the zero start at identical tolerances.

Tolerances: forward outputs within 1e-5 and gradients within 1e-4 (relative 2-norm per
parameter block) of the FP64 oracle -- the GPU computes in FP32; projections of basis
combinations within 1e-12; a warm-started solve meets the same Newton gates as the zero
start, so the two solutions agree to the step gate (A within 1e-6 relative).
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import mlp_oracle as M
from femm_gpu_b200 import learned, meshes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / max(
        np.linalg.norm(np.asarray(b, np.float64)), 1e-300)


def test_mlp_forward_and_gradient_match_cpu_oracle(gpu):
    I, H, O, B = 4, 256, 64, 96
    net = learned.Mlp(I, H, O, seed=7)
    p = net.get_parameters()
    assert p.size == H * I + H + H * H + H + O * H + O == net.parameter_count
    rng = np.random.default_rng(1)
    x = rng.normal(size=(B, I)).astype(np.float32)
    t = rng.normal(size=(B, O)).astype(np.float32)
    y = net.forward(x)
    y64, _ = M.forward(p, x, I, H, O)
    assert rel(y, y64) <= 1e-5
    loss, g = net.loss_gradient(x, t)
    loss64, g64 = M.loss_gradient(p, x, t, I, H, O)
    assert abs(loss - loss64) <= 1e-5 * loss64
    o = 0
    for n in (H * I, H, H * H, H, O * H, O):
        assert rel(g[o:o + n], g64[o:o + n]) <= 1e-4, (o, n)
        o += n


def test_mlp_training_is_reproducible_and_learns(gpu):
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, size=(512, 4)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 1], x[:, 2] ** 2 - x[:, 3], x[:, 0] * x[:, 3]], axis=1)
    t = t.astype(np.float32)
    runs = []
    for _ in range(2):
        net = learned.Mlp(4, 64, 3, seed=3)
        l0, _ = net.loss_gradient(x, t)
        loss = net.train(x, t, epochs=150, batch=64, lr=3e-3, seed=4)
        runs.append((l0, loss, net.get_parameters()))
    assert runs[0][1] < 0.02 * runs[0][0]
    assert runs[0][1] == runs[1][1] and np.array_equal(runs[0][2], runs[1][2])
    # the trained loss is the oracle's loss of the trained parameters
    loss64, _ = M.loss_gradient(runs[0][2], x, t, 4, 64, 3)
    assert abs(runs[0][1] - loss64) <= 1e-4 * loss64


def plunger():
    return meshes.axisymmetric_plunger(mr=24, mz=48)


def test_reduced_basis_projection_round_trip(gpu):
    model = plunger()
    plan = fg.Plan(model)
    rng = np.random.default_rng(5)
    q, _ = np.linalg.qr(rng.normal(size=(model.node_count, 12)))
    basis = q.T.copy()
    mean = rng.normal(size=model.node_count)
    wm = learned.WarmModel(plan, mean, basis)
    c = rng.normal(size=(5, 12))
    a = mean + c @ basis
    np.testing.assert_allclose(wm.project(a), c, rtol=0, atol=1e-12 * np.abs(c).max() * model.node_count)


@pytest.fixture(scope="module")
def trained():
    model = plunger()
    plan = fg.Plan(model)
    rng = np.random.default_rng(11)
    train = rng.uniform(-30, 30, size=(256, 2))
    ws = learned.LearnedWarmStart(plan, current_scale=30.0, rank=16, hidden=64, seed=5)
    ws.fit(train, pod_samples=128, epochs=300, batch=64, lr=3e-3)
    held = np.random.default_rng(12).uniform(-30, 30, size=(48, 2))
    return model, plan, ws, held


def test_learned_warm_start_gains_over_zero_start(gpu, trained):
    model, plan, ws, held = trained
    assert ws.stats["pod_energy"] > 0.999
    zero = plan.solve(held)
    warm = ws.solve(held)
    assert all(s == 0 for s in zero.status) and all(s == 0 for s in warm.status)
    assert all(i.warm_start in (1, 2) for i in warm.info)
    used = sum(1 for i in warm.info if i.warm_start == 1)
    assert used >= 0.9 * len(held)
    zn = sum(i.iterations for i in zero.info)
    wn = sum(i.iterations for i in warm.info)
    zl = sum(i.linear_iterations for i in zero.info)
    wl = sum(i.linear_iterations for i in warm.info)
    assert wn < zn and wl < zl, (wn, zn, wl, zl)
    for k in range(len(held)):
        assert rel(warm.a[k], zero.a[k]) <= 1e-6
        assert rel(warm.flux[k], zero.flux[k]) <= 1e-6


def test_guard_rejects_a_bad_guess_and_matches_the_zero_start(gpu, trained):
    model, plan, ws, held = trained
    # the same network with its coefficient scale blown up: a guess far worse than zero
    w = ws.warm
    bad = learned.WarmModel(plan, w.mean, w.basis, ws.mlp, *w._keep[:2], w._keep[2],
                            w._keep[3] * 1e4)
    guard = learned.LearnedWarmStart(plan, 30.0)
    guard.warm = bad
    got = guard.solve(held[:6])
    zero = plan.solve(held[:6])
    assert all(i.warm_start == 2 for i in got.info)
    for k in range(6):
        assert got.info[k].iterations == zero.info[k].iterations
        assert np.array_equal(got.a[k], zero.a[k])
    # a supplied (unguarded) warm start is reported as used
    plain = plan.solve(held[:2], warm=zero.a[:2])
    assert all(i.warm_start == 1 for i in plain.info)


@pytest.mark.parametrize("precision", [0, 1])
def test_pcg_from_iterate_matches_oracle(gpu, precision):
    """FG_PLAN_PCG_FROM_ITERATE: the inner PCG solves for the correction from the current
    iterate under the same acceptance rule, so the Newton solution matches the oracle's
    (zero-start PCG) within cond(K) x 1e-10: A within 2e-8, flux within 1e-8."""
    import oracle as O
    model = meshes.square_nonlinear(m=24, seed=4)
    currents = meshes.seeded_currents(3, 3, 20.0, seed=9)
    plan = fg.Plan(model, from_iterate=True, precision=precision)
    got = plan.solve(currents)
    a, b1, b2, flux, info = O.solve_batch(model, currents)
    for k in range(3):
        assert got.info[k].status == info[k].status == 0
        assert abs(got.info[k].iterations - info[k].iterations) <= 1
        assert rel(got.a[k], a[k]) <= 2e-8
        assert rel(got.flux[k], flux[k]) <= 1e-8
    plain = fg.Plan(model).solve(currents)
    assert sum(i.linear_iterations for i in got.info) < sum(i.linear_iterations for i in plain.info)
