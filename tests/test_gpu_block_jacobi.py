"""GPU parity of the block-Jacobi preconditioner (8- and 32-row blocks) against the oracle.

Tolerances are those of the Jacobi PCG and Newton tests: true residual within the
tolerance, x within 1e-6 of the oracle's PCG at 1e-10, iteration counts within 15 %;
Newton solves with the same status and iteration count, A within 1e-9 and flux linkage
within 1e-8 (relative 2-norm).  The mixed form (FP32 inner PCG with FP32 block inverses)
is held to the mixed-form bounds against the FP64 oracle: A 2e-8, flux 1e-8.
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def residual(sysm, x, rhs):
    ax = np.zeros(sysm.rows)
    for r in range(sysm.rows):
        sl = slice(sysm.off[r], sysm.off[r + 1])
        ax[r] = np.dot(sysm.val[sl], x[sysm.col[sl]])
    return np.linalg.norm(rhs - ax) / np.linalg.norm(rhs)


def assembled(m=48, seed=11):
    model = meshes.square_nonlinear(m=m, seed=seed)
    rng = np.random.default_rng(3)
    a = rng.normal(size=model.node_count) * 1e-3
    a[model.dir_nodes] = 0.0
    return model, O.assemble(model, a, [4.0, -7.0, 2.0], 1)


@pytest.mark.parametrize("bs", [8, 32])
def test_block_pcg_matches_oracle(gpu, bs):
    model, sysm = assembled()
    plan = fg.Plan(model, preconditioner=1, block_size=bs)
    with O.preconditioner(1, bs):
        s_or, x_or, it_or, _ = O.pcg(sysm, tol=1e-10)
    x, info = plan.pcg(sysm.val[None, :], sysm.rhs[None, :], tol=1e-10)
    assert info[0].status == 0 and s_or == 0
    assert residual(sysm, x[0], sysm.rhs) <= 1e-10 * (1 + 1e-9)
    assert rel(x[0], x_or) <= 1e-6
    assert abs(info[0].iterations - it_or) <= max(3, 0.15 * it_or)
    assert plan.last_timing().block_fallbacks == 0
    # per-item operators (scaled copies) and a shared operator with several right-hand sides
    k = 5
    vals = np.stack([sysm.val * (1.0 + 0.25 * i) for i in range(k)])
    rhs = np.stack([sysm.rhs * (i - 2.5) for i in range(k)])
    x, info = plan.pcg(vals, rhs, tol=1e-10)
    # Each item against the oracle's block PCG on the same (scaled) system: two answers
    # that both meet ||b - Ax|| <= 1e-10 ||b|| may differ by cond(A) * 1e-10, so x is
    # compared item by item, not against a rescaled single solution, within 1e-5 (the
    # scaled items stop at different iterations of a recurrence whose rounding differs).
    with O.preconditioner(1, bs):
        for i in range(k):
            item = O.csr_system(sysm.off, sysm.col, vals[i], rhs[i])
            s_i, x_i, it_i, _ = O.pcg(item, tol=1e-10)
            assert info[i].status == 0 == s_i
            assert residual(item, x[i], rhs[i]) <= 1e-10 * (1 + 1e-9)
            assert rel(x[i], x_i) <= 1e-5
        x, info = plan.pcg(sysm.val, rhs[:3], tol=1e-10, shared=True)
        for i in range(3):
            s_i, x_i, it_i, _ = O.pcg(sysm, rhs=rhs[i], tol=1e-10)
            assert info[i].status == 0 == s_i
            assert rel(x[i], x_i) <= 1e-5


def test_unusable_block_falls_back_like_the_oracle(gpu):
    model, sysm = assembled(m=32, seed=5)
    val = sysm.val.copy()
    r = 8  # row 8, first row of block 1
    k = next(k for k in range(sysm.off[r], sysm.off[r + 1]) if sysm.col[k] == r + 1)
    val[k] *= 1.0 + 1e-9
    pert = O.csr_system(sysm.off, sysm.col, val, sysm.rhs)
    inv, fb = O.block_jacobi(pert, 8)
    assert fb == 1 and np.isnan(inv[1, 0])
    with O.preconditioner(1, 8):
        s_or, x_or, it_or, _ = O.pcg(pert, tol=1e-10)
    plan = fg.Plan(model, preconditioner=1, block_size=8)
    x, info = plan.pcg(val[None, :], sysm.rhs[None, :], tol=1e-10)
    assert info[0].status == s_or == 0
    assert plan.last_timing().block_fallbacks == 1
    assert rel(x[0], x_or) <= 1e-6


@pytest.mark.parametrize("bs", [8, 32])
def test_newton_block_jacobi_matches_oracle(gpu, bs):
    model = meshes.square_nonlinear(m=24, seed=4)
    currents = meshes.seeded_currents(3, 3, 20.0, seed=9)
    plan = fg.Plan(model, preconditioner=1, block_size=bs)
    got = plan.solve(currents)
    with O.preconditioner(1, bs):
        a, b1, b2, flux, info = O.solve_batch(model, currents)
    for k in range(3):
        assert got.info[k].status == info[k].status == 0
        assert got.info[k].iterations == info[k].iterations
        assert rel(got.a[k], a[k]) <= 1e-9
        assert rel(got.flux[k], flux[k]) <= 1e-8
    t = plan.last_timing()
    assert t.block_inverses > 0 and t.block_fallbacks == 0


def test_mixed_precision_with_32_row_blocks(gpu):
    model = meshes.square_nonlinear(m=40, seed=6)
    currents = meshes.seeded_currents(4, 3, 20.0, seed=12)
    plan = fg.Plan(model, preconditioner=1, block_size=32, precision=1)
    got = plan.solve(currents)
    a, b1, b2, flux, info = O.solve_batch(model, currents)
    for k in range(4):
        assert got.info[k].status == info[k].status == 0
        assert rel(got.a[k], a[k]) <= 2e-8
        assert rel(got.flux[k], flux[k]) <= 1e-8
    assert plan.last_timing().mixed_fallbacks == 0


def test_32_row_blocks_chunk_at_16_items(gpu):
    model = meshes.square_nonlinear(m=16, seed=2)
    currents = meshes.seeded_currents(20, 3, 20.0, seed=3)
    plan = fg.Plan(model, preconditioner=1, block_size=32)
    got = plan.solve(currents)
    with O.preconditioner(1, 32):
        a, _, _, flux, info = O.solve_batch(model, currents)
    for k in range(20):
        assert got.info[k].status == info[k].status == 0
        assert rel(got.a[k], a[k]) <= 1e-9
    sysm = O.assemble(model, np.zeros(model.node_count), currents[0], 0)
    with pytest.raises(fg.FgError) as e:
        plan.pcg(np.tile(sysm.val, (17, 1)), np.tile(sysm.rhs, (17, 1)))
    assert e.value.status == fg.capi.UNSUPPORTED_FEATURE
