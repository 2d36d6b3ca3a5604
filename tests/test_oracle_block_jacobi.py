"""The oracle's block-Jacobi preconditioner (block_jacobi_preconditioner.cu:72-167 and
pcg_device.cuh:62-79 of the reference) on the CPU.

The reference tests its block mode on 1/7/8/9/31/32/33/67/4097 unknowns, FEM grids,
factorization failure and the diagonal fallback (PERFORMANCE.md, "Selectable block
preconditioner"); the same cases are checked here against numpy: every usable block's
stored inverse times the block is the identity, unusable blocks carry NaN in their first
entry, and the block-preconditioned PCG meets the same true-residual gate as Jacobi.
"""
import numpy as np
import pytest

import oracle as O
from femm_gpu_b200 import meshes


def laplacian_csr(n, seed=0):
    """SPD test operator: 1D Laplacian with random positive couplings to row i +- 3."""
    rng = np.random.default_rng(seed)
    rows = [dict() for _ in range(n)]
    for i in range(n):
        rows[i][i] = 0.0
    for i in range(n):
        for d in (1, 3):
            j = i + d
            if j < n:
                w = rng.uniform(0.5, 2.0)
                rows[i][j] = rows[i].get(j, 0.0) - w
                rows[j][i] = rows[j].get(i, 0.0) - w
                rows[i][i] += w
                rows[j][j] += w
    for i in range(n):
        rows[i][i] += rng.uniform(0.01, 0.1)
    off, col, val = [0], [], []
    for i in range(n):
        for j in sorted(rows[i]):
            col.append(j)
            val.append(rows[i][j])
        off.append(len(col))
    return np.array(off), np.array(col), np.array(val)


def dense(sysm):
    A = np.zeros((sysm.rows, sysm.rows))
    for r in range(sysm.rows):
        for k in range(sysm.off[r], sysm.off[r + 1]):
            A[r, sysm.col[k]] = sysm.val[k]
    return A


def check_inverses(sysm, bs):
    inv, fb = O.block_jacobi(sysm, bs)
    A = dense(sysm) if sysm.rows <= 5000 else None
    n = sysm.rows
    for b in range(inv.shape[0]):
        first, w = b * bs, min(bs, n - b * bs)
        binv = inv[b].reshape(bs, bs).T  # [i][j]
        if np.isnan(binv[0, 0]):
            continue
        assert not binv[w:, :].any() and not binv[:, w:].any()
        if A is not None:
            blk = A[first:first + w, first:first + w]
            np.testing.assert_allclose(binv[:w, :w] @ blk, np.eye(w), atol=1e-11)
    return inv, fb


@pytest.mark.parametrize("n", [1, 7, 8, 9, 31, 32, 33, 67, 4097])
@pytest.mark.parametrize("bs", [8, 32])
def test_block_inverses_and_pcg_sizes(n, bs):
    off, col, val = laplacian_csr(n, seed=n)
    rng = np.random.default_rng(n + 1)
    sysm = O.csr_system(off, col, val, rng.normal(size=n))
    inv, fb = check_inverses(sysm, bs)
    assert fb == 0 and not np.isnan(inv).any()
    with O.preconditioner(1, bs):
        st, x, its, res = O.pcg(sysm, tol=1e-12)
    assert st == 0
    A = dense(sysm)
    assert np.linalg.norm(sysm.rhs - A @ x) <= 1e-12 * np.linalg.norm(sysm.rhs) * (1 + 1e-9)
    np.testing.assert_allclose(x, np.linalg.solve(A, sysm.rhs), rtol=0, atol=1e-8 * np.abs(x).max())


def test_fem_grid_blocks_are_exact_inverses():
    model = meshes.square_linear(m=64)
    sysm = O.assemble(model, np.zeros(model.node_count), [12.0], 0)
    for bs in (8, 32):
        inv, fb = check_inverses(sysm, bs)
        assert fb == 0
        with O.preconditioner(1, bs):
            st, x, its, res = O.pcg(sysm)
        st0, x0, its0, res0 = O.pcg(sysm)
        assert st == 0 and st0 == 0
        assert np.linalg.norm(x - x0) <= 1e-6 * np.linalg.norm(x0)


def test_unusable_blocks_fall_back_to_the_diagonal():
    off, col, val = laplacian_csr(40, seed=5)
    val = val.copy()
    # (a) asymmetric coupling inside block 0 (rows 0..7)
    k01 = next(k for k in range(off[0], off[1]) if col[k] == 1)
    val[k01] *= 1.0 + 1e-9
    # (b) failed pivot in block 2 (rows 16..23): a coupling larger than the diagonals
    k = next(k for k in range(off[16], off[17]) if col[k] == 17)
    k2 = next(k for k in range(off[17], off[18]) if col[k] == 16)
    val[k] = val[k2] = -10.0 * max(val[off[16]:off[17]].max(), 1.0)
    sysm = O.csr_system(off, col, val, np.ones(40))
    inv, fb = O.block_jacobi(sysm, 8)
    assert fb == 2
    assert np.isnan(inv[0, 0]) and not np.isnan(inv[1, 0]) and np.isnan(inv[2, 0])
    assert not inv[0, 1:].any() and not inv[2, 1:].any()
    # (c) a subnormal reciprocal diagonal marks its block
    val3 = np.asarray(laplacian_csr(16, seed=1)[2]).copy()
    off3, col3, _ = laplacian_csr(16, seed=1)
    kd = next(k for k in range(off3[9], off3[10]) if col3[k] == 9)
    val3[kd] = 1e308
    inv3, fb3 = O.block_jacobi(O.csr_system(off3, col3, val3), 8)
    assert fb3 == 1 and not np.isnan(inv3[0, 0]) and np.isnan(inv3[1, 0])


def test_fallback_block_still_solves():
    off, col, val = laplacian_csr(64, seed=8)
    val = val.copy()
    k01 = next(k for k in range(off[0], off[1]) if col[k] == 1)
    val[k01] *= 1.0 + 1e-9  # block 0 unusable, the operator still (almost) symmetric
    sysm = O.csr_system(off, col, val, np.linspace(-1.0, 1.0, 64))
    with O.preconditioner(1, 8):
        st, x, its, res = O.pcg(sysm, tol=1e-10)
    assert st == 0
    A = dense(sysm)
    assert np.linalg.norm(sysm.rhs - A @ x) <= 1e-10 * np.linalg.norm(sysm.rhs) * (1 + 1e-9)


def test_newton_with_block_jacobi_matches_jacobi():
    model = meshes.square_nonlinear(m=20, seed=3)
    currents = meshes.seeded_currents(2, 3, 20.0, seed=5)
    a0, _, _, f0, i0 = O.solve_batch(model, currents)
    with O.preconditioner(1, 8):
        a1, _, _, f1, i1 = O.solve_batch(model, currents)
    for k in range(2):
        assert i0[k].status == 0 and i1[k].status == 0
        assert np.linalg.norm(a1[k] - a0[k]) <= 1e-7 * np.linalg.norm(a0[k])
        assert np.linalg.norm(f1[k] - f0[k]) <= 1e-7 * np.linalg.norm(f0[k])
