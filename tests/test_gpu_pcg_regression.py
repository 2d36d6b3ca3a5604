"""The reference's PCG regression and determinism suite, through the C ABI.

Systems (gpu_solver/tests/native/pcg_regression.cu:13-187): the five-point stencil on a
side x side grid (side 67 and 129: rows spread over many CTAs with uneven tails and
couplings across CTA boundaries), off-diagonal -1, diagonal 4.05 + 0.01 (row mod 7), and
the manufactured solution x_i = sin(0.17 i) + 0.3 cos(0.071 i).  Checks:
* one solve: true residual ||b - A x|| <= 1.01e-10 ||b|| and max |x - exact| < 1e-8;
* batch widths 1, 2, 4, 5 and 32, shared operator, right-hand sides scaled per item (item
  1 zero, odd items -0.75, even items 1 + 0.1 item): every item within the residual gate;
  then a distinct operator per item (values and diagonal x (1 + 0.2 item)): the same;
* a single solve repeated is bitwise identical with the same iteration count;
* statuses: a zero iteration budget cannot pass, a zero right-hand side passes without an
  iteration, a negative tolerance is INVALID_ARGUMENT, a NaN right-hand side is
  NUMERICAL_NONFINITE, a negative diagonal is LINEAR_SOLVE_BREAKDOWN, and when both occur
  the earlier row decides;
* failed, zero and live right-hand sides in one launch: the live ones still pass;
* a diagonal system of 1e308 entries (the reciprocal is subnormal, so the Jacobi step
  divides) still meets the residual gate;
* 100 repeated nonlinear solves are bitwise identical and the device's free memory does
  not shrink (self_test.cu:296-311).
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
from femm_gpu_b200 import meshes

pytestmark = pytest.mark.gpu

GATE = 1.01e-10


def five_point(side):
    n = side * side
    rows, cols, vals = [], [], []
    diag = 4.05 + 0.01 * (np.arange(n) % 7)
    for r in range(n):
        nb = []
        if r >= side:
            nb.append((r - side, -1.0))
        if r % side:
            nb.append((r - 1, -1.0))
        nb.append((r, diag[r]))
        if r % side != side - 1:
            nb.append((r + 1, -1.0))
        if r < n - side:
            nb.append((r + side, -1.0))
        for c, v in nb:
            rows.append(r)
            cols.append(c)
            vals.append(v)
    ro = np.zeros(n + 1, np.int32)
    np.add.at(ro, np.asarray(rows) + 1, 1)
    ro = np.cumsum(ro).astype(np.int32)
    i = np.arange(n)
    exact = np.sin(0.17 * i) + 0.3 * np.cos(0.071 * i)
    col, val = np.asarray(cols, np.int32), np.asarray(vals)
    return ro, col, val, diag, exact


def multiply(ro, col, val, x):
    rows = np.repeat(np.arange(ro.size - 1), np.diff(ro))
    return np.bincount(rows, weights=val * x[col], minlength=ro.size - 1)


def verified(ro, col, val, rhs, x, info):
    if info.status != fg.capi.OK or not np.all(np.isfinite(x)):
        return False
    return np.linalg.norm(multiply(ro, col, val, x) - rhs) <= GATE * np.linalg.norm(rhs)


@pytest.mark.parametrize("side", [67, 129])
def test_manufactured_five_point_systems(gpu, side):
    ro, col, val, diag, exact = five_point(side)
    n = exact.size
    rhs = multiply(ro, col, val, exact)
    x, info = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=1e-10, maxit=2000)
    assert verified(ro, col, val, rhs, x[0], info[0])
    assert np.max(np.abs(x[0] - exact)) < 1e-8
    for width in (1, 2, 4, 5, 32):
        factors = [0.0 if i == 1 else (-0.75 if i % 2 else 1.0 + 0.1 * i) for i in range(width)]
        rhs_w = np.stack([f * rhs for f in factors])
        xs, infos = fg.csr_pcg(ro, col, val, diag, rhs_w, tol=1e-10, maxit=2000, shared=True)
        for i in range(width):
            assert verified(ro, col, val, rhs_w[i], xs[i], infos[i]), (width, i)
        scale = np.array([1.0 + 0.2 * i for i in range(width)])
        vals_w = scale[:, None] * val[None, :]
        diags_w = scale[:, None] * diag[None, :]
        xs, infos = fg.csr_pcg(ro, col, vals_w, diags_w, rhs_w, tol=1e-10, maxit=2000)
        for i in range(width):
            assert verified(ro, col, vals_w[i], rhs_w[i], xs[i], infos[i]), (width, i, "distinct")
        again, ainfo = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=1e-10, maxit=2000)
        assert np.array_equal(again, x) and ainfo[0].iterations == info[0].iterations
    # statuses
    _, i0 = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=1e-10, maxit=0)
    assert i0[0].status == fg.capi.LINEAR_SOLVE_NOT_CONVERGED
    z, iz = fg.csr_pcg(ro, col, val, diag, np.zeros((1, n)), tol=1e-10, maxit=0)
    assert iz[0].status == fg.capi.OK and not z.any()
    _, ineg = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=-1.0, maxit=10)
    assert ineg[0].status == fg.capi.INVALID_ARGUMENT
    nan17 = rhs.copy()
    nan17[17] = np.nan
    _, inan = fg.csr_pcg(ro, col, val, diag, nan17[None, :], tol=1e-10, maxit=10)
    assert inan[0].status == fg.capi.NUMERICAL_NONFINITE
    bad = diag.copy()
    bad[19] = -1.0
    _, ib = fg.csr_pcg(ro, col, val, bad, rhs[None, :], tol=1e-10, maxit=10)
    assert ib[0].status == fg.capi.LINEAR_SOLVE_BREAKDOWN
    _, ib = fg.csr_pcg(ro, col, val, bad, nan17[None, :], tol=1e-10, maxit=10)
    assert ib[0].status == fg.capi.NUMERICAL_NONFINITE  # row 17 comes before row 19
    nanlast = rhs.copy()
    nanlast[n - 1] = np.nan
    _, ib = fg.csr_pcg(ro, col, val, bad, nanlast[None, :], tol=1e-10, maxit=10)
    assert ib[0].status == fg.capi.LINEAR_SOLVE_BREAKDOWN  # row 19 comes before the last row
    # failed, zero and live right-hand sides in one cooperative launch
    xs, infos = fg.csr_pcg(ro, col, val, diag, np.stack([rhs, nanlast, np.zeros(n), rhs]), tol=1e-10,
                           maxit=2000, shared=True)
    assert infos[1].status == fg.capi.NUMERICAL_NONFINITE and infos[2].status == fg.capi.OK
    assert verified(ro, col, val, rhs, xs[0], infos[0]) and verified(ro, col, val, rhs, xs[3], infos[3])
    # extreme scale: the reciprocal of 1e308 is subnormal, so the Jacobi step divides
    ro_d = np.arange(n + 1, dtype=np.int32)
    col_d = np.arange(n, dtype=np.int32)
    big = np.full(n, 1e308)
    xs, infos = fg.csr_pcg(ro_d, col_d, big, big, np.ones((1, n)), tol=1e-10, maxit=10)
    assert verified(ro_d, col_d, big, np.ones(n), xs[0], infos[0])


def test_hundred_repeats_bitwise_and_no_memory_growth(gpu):
    import torch

    model = meshes.square_nonlinear(m=20, seed=8)
    currents = meshes.seeded_currents(2, 3, 20.0, seed=1)
    plan = fg.Plan(model)
    first = plan.solve(currents)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(100):
        r = plan.solve(currents)
        for f in ("a", "b1", "b2", "flux"):
            assert np.array_equal(getattr(r, f), getattr(first, f))
        assert [i.iterations for i in r.info] == [i.iterations for i in first.info]
        assert [i.linear_iterations for i in r.info] == [i.linear_iterations for i in first.info]
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after >= free_before


def test_grid_wait_that_runs_out_ends_the_launch_cleanly(gpu):
    """Every grid-wide wait of the PCG is bounded (the reference bounds its device loops,
    pcg_kernels.cu:555-566).  With a 1 ns bound the first wait runs out: every CTA
    returns, the call reports INTERNAL_ERROR, and with the default bound restored the same
    solve passes on the same context."""
    ro, col, val, diag, exact = five_point(129)  # 16,641 rows: a launch of many CTAs
    rhs = multiply(ro, col, val, exact)
    previous = fg.capi.set_wait_limit_ns(1)
    try:
        with pytest.raises(fg.FgError) as err:
            fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=1e-10, maxit=2000)
        assert err.value.status == fg.capi.INTERNAL_ERROR
        plan = fg.Plan(meshes.square_nonlinear(m=40, seed=3))
        with pytest.raises(fg.FgError) as err:
            plan.solve(meshes.seeded_currents(2, 3, 20.0, seed=5))
        assert err.value.status == fg.capi.INTERNAL_ERROR
    finally:
        assert fg.capi.set_wait_limit_ns(previous) == 1
    x, info = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=1e-10, maxit=2000)
    assert verified(ro, col, val, rhs, x[0], info[0])
    r = plan.solve(meshes.seeded_currents(2, 3, 20.0, seed=5))
    assert r.status == [0, 0]
