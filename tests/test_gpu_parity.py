"""GPU parity: libfemmgpu (through the C ABI) against the CPU oracle.

Tolerances:
* assembly: |gpu - oracle| <= 1e-12 * max|oracle| + 5e-11 * |oracle| (the reference's
  NearMixed(1e-12, 5e-11) host/device gate, protocol_contract_tests.cu:963-1013, with the
  absolute part scaled to the system's magnitude because the models are in SI units);
  repeated assembly is bitwise identical;
* PCG: the true residual ||b - A x|| / ||b|| <= tolerance, x within 1e-6 (relative
  2-norm) of the oracle's PCG on the same system at tolerance 1e-10, iteration counts
  within 15 %;
* Newton solves: same status and Newton iteration count; A within 1e-9 and flux linkage
  within 1e-8 relative 2-norm of the oracle; B within 1e-8 relative to max|B|;
* stock-FEMM fixtures: flux within 1e-10 (strips) / 1e-3 (axisymmetric) as the reference's
  own tests require.
"""
import json
import os

import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from conftest import GOLDEN
from femm_gpu_b200 import artifact, meshes
from test_oracle_fixtures import two_circuit, unit_square

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


# ----------------------------------------------------------------------------- PCG
def test_pcg_known_answers(gpu):
    ro, col = [0, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2]
    val = np.array([4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 3.0])
    diag = np.array([4.0, 4.0, 3.0])
    x, info = fg.csr_pcg(ro, col, val, diag, [[2.0, 4.0, 7.0]], tol=1e-13, maxit=64)
    assert info[0].status == 0
    np.testing.assert_allclose(x[0], [1.0, 2.0, 3.0], rtol=1e-13)
    # shared-operator two-RHS launch (self_test.cu:55-76): exact answers
    x, info = fg.csr_pcg(ro, col, val, diag, [[2.0, 4.0, 7.0], [4.0, 8.0, 14.0]], shared=True)
    assert [i.status for i in info] == [0, 0]
    assert np.array_equal(x[0], [1.0, 2.0, 3.0]) and np.array_equal(x[1], [2.0, 4.0, 6.0])
    # per-item operators
    x, info = fg.csr_pcg(ro, col, np.stack([val, 2 * val]), np.stack([diag, 2 * diag]),
                         [[2.0, 4.0, 7.0], [4.0, 8.0, 14.0]])
    np.testing.assert_allclose(x, [[1, 2, 3], [1, 2, 3]], rtol=1e-13)
    # 513 rows: reduction tail beyond one block width, identity operator, exact
    n = 513
    rhs = np.array([(i % 11) - 5 for i in range(n)], dtype=float)
    x, info = fg.csr_pcg(np.arange(n + 1), np.arange(n), np.ones((2, n)), np.ones((2, n)), [rhs, rhs],
                         maxit=16)
    assert [i.status for i in info] == [0, 0] and np.array_equal(x[0], rhs) and np.array_equal(x[1], rhs)
    # indefinite -> LINEAR_SOLVE_BREAKDOWN (self_test.cu:125-137)
    x, info = fg.csr_pcg([0, 1], [0], [-1.0], [-1.0], [[1.0]], maxit=8)
    assert info[0].status == fg.capi.LINEAR_SOLVE_BREAKDOWN
    # iteration budget 0 -> LINEAR_SOLVE_NOT_CONVERGED; infinite tolerance -> INVALID_ARGUMENT
    x, info = fg.csr_pcg(ro, col, val, diag, [[2.0, 4.0, 7.0]], tol=1e-13, maxit=0)
    assert info[0].status == fg.capi.LINEAR_SOLVE_NOT_CONVERGED
    x, info = fg.csr_pcg(ro, col, val, diag, [[2.0, 4.0, 7.0]], tol=float("inf"), maxit=8)
    assert info[0].status == fg.capi.INVALID_ARGUMENT
    # a zero RHS is an exact zero solution; tiny RHS are solved, not accepted at x = 0
    x, info = fg.csr_pcg(ro, col, val, diag, [[0.0, 0.0, 0.0], [2e-200, 4e-200, 7e-200]], tol=1e-13,
                         shared=True)
    assert info[0].status == 0 and info[0].iterations == 0 and not x[0].any()
    assert info[1].status == 0 and info[1].iterations > 0
    np.testing.assert_allclose(x[1], [1e-200, 2e-200, 3e-200], rtol=1e-12)
    # non-finite RHS -> NUMERICAL_NONFINITE, isolated from its batch neighbour
    x, info = fg.csr_pcg(ro, col, val, diag, [[np.nan, 1.0, 1.0], [2.0, 4.0, 7.0]], shared=True)
    assert info[0].status == fg.capi.NUMERICAL_NONFINITE and info[1].status == 0


def test_pcg_matches_oracle_on_assembled_system(gpu):
    model = meshes.square_nonlinear(m=48, seed=11)
    rng = np.random.default_rng(3)
    a = rng.normal(size=model.node_count) * 1e-3
    a[model.dir_nodes] = 0.0
    sysm = O.assemble(model, a, [4.0, -7.0, 2.0], 1)
    plan = fg.Plan(model)
    # Two solutions that each meet ||b - Ax|| <= tol ||b|| may differ by up to cond(A) * tol,
    # so the solutions are compared at the production tolerance only.
    for tol in (1e-6, 1e-10):
        s_or, x_or, it_or, _ = O.pcg(sysm, tol=tol)
        x, info = plan.pcg(sysm.val[None, :], sysm.rhs[None, :], tol=tol)
        assert info[0].status == 0 and s_or == 0
        # true residual of the GPU answer, recomputed in numpy
        A = np.zeros(sysm.rows)
        for r in range(sysm.rows):
            sl = slice(sysm.off[r], sysm.off[r + 1])
            A[r] = np.dot(sysm.val[sl], x[0][sysm.col[sl]])
        assert np.linalg.norm(sysm.rhs - A) <= tol * np.linalg.norm(sysm.rhs) * (1 + 1e-9)
        if tol == 1e-10:
            assert rel(x[0], x_or) <= 1e-6
        # Same recurrence, different rounding (FMA, tree reductions): CG on this
        # 1000:1 contrast operator drifts by some percent in iteration count.
        assert abs(info[0].iterations - it_or) <= max(3, 0.15 * it_or)


# ----------------------------------------------------------------------------- assembly
def assembly_models():
    return [meshes.square_nonlinear(m=16, seed=2), meshes.square_linear(m=12),
            meshes.periodic_strip(m=10), meshes.periodic_strip(m=10, antiperiodic=True),
            meshes.axisymmetric_plunger(mr=10, mz=16)]


@pytest.mark.parametrize("idx", range(5))
def test_assembly_matches_oracle(gpu, idx):
    model = assembly_models()[idx]
    plan = fg.Plan(model)
    ro, col, *_ = plan.symbolic()
    rng = np.random.default_rng(idx)
    states = rng.normal(size=(3, model.node_count)) * 3e-3
    states[:, model.dir_nodes] = 0.0
    if model.problem_type == 1:
        states *= model.xy[:, 0][None, :] / model.xy[:, 0].max()
    currents = rng.uniform(-15, 15, size=(3, model.circuit_count))
    for use_newton in (0, 1):
        vals, diag, rhs = plan.assemble(states, currents, use_newton)
        for k in range(3):
            ref = O.assemble(model, states[k], currents[k], use_newton)
            assert np.array_equal(ro, ref.off) and np.array_equal(col, ref.col)
            for got, exp in ((vals[k], ref.val), (diag[k], ref.diag), (rhs[k], ref.rhs)):
                tol = 1e-12 * np.max(np.abs(exp)) + 5e-11 * np.abs(exp)
                assert np.all(np.abs(got - exp) <= tol), np.max(np.abs(got - exp) / (np.abs(exp) + 1e-300))
        again = plan.assemble(states, currents, use_newton)
        for x, y in zip((vals, diag, rhs), again):
            assert np.array_equal(x, y)


# ----------------------------------------------------------------------------- Newton
def check_solve(model, currents, res_tol_a=1e-9, res_tol_flux=1e-8, warm=None):
    plan = fg.Plan(model)
    got = plan.solve(currents, warm=warm)
    a, b1, b2, flux, info = O.solve_batch(model, currents, warm=warm)
    for k in range(len(info)):
        assert got.info[k].status == info[k].status, (k, got.info[k].status, info[k].status)
        if info[k].status != 0:
            continue
        assert got.info[k].iterations == info[k].iterations
        assert rel(got.a[k], a[k]) <= res_tol_a, rel(got.a[k], a[k])
        assert rel(got.flux[k], flux[k]) <= res_tol_flux, rel(got.flux[k], flux[k])
        bmax = max(np.max(np.abs(b1[k])), np.max(np.abs(b2[k])))
        assert np.max(np.abs(got.b1[k] - b1[k])) <= 1e-8 * bmax
        assert np.max(np.abs(got.b2[k] - b2[k])) <= 1e-8 * bmax
    return plan, got


def test_newton_nonlinear_square_matches_oracle(gpu):
    model = meshes.square_nonlinear(m=24, seed=4)
    currents = meshes.seeded_currents(3, 3, 20.0, seed=9)
    check_solve(model, currents)


def test_newton_linear_square_matches_oracle(gpu):
    check_solve(meshes.square_linear(m=32), np.array([[10.0], [-3.0]]))


def test_newton_axisymmetric_matches_oracle(gpu):
    check_solve(meshes.axisymmetric_plunger(mr=12, mz=24), meshes.seeded_currents(2, 2, 30.0, 5))


@pytest.mark.parametrize("name,rtol", [("periodic_strip", 1e-10), ("antiperiodic_strip", 1e-10),
                                       ("axisymmetric_coil", 1e-3)])
def test_stock_femm_fixtures(gpu, name, rtol):
    expected = json.load(open(os.path.join(GOLDEN, "expected.json")))[name]["flux_linkage_Wb"]
    model, currents = artifact.read_artifact(open(os.path.join(GOLDEN, name + ".gpu.json")).read())
    plan, got = check_solve(model, currents[None, :])
    assert got.info[0].status == 0
    assert abs(got.flux[0, 0] - expected) <= rtol * abs(expected)
    if model.con_a.size:
        pair = got.a[0, model.con_b] - model.con_sign * got.a[0, model.con_a]
        assert np.max(np.abs(pair)) <= 1e-15 * np.max(np.abs(got.a[0]))


def test_known_answers_unit_square_and_two_circuits(gpu):
    plan = fg.Plan(unit_square())
    r = plan.solve([[12.0], [-12.0]])
    assert r.status == [0, 0]
    np.testing.assert_allclose(r.a[0], [0, 0, 0, 0, 1.0], atol=1e-12)
    np.testing.assert_allclose(r.b1[0], [2, 0, -2, 0], atol=1e-12)
    np.testing.assert_allclose(r.b2[0], [0, 2, 0, -2], atol=1e-12)
    assert r.flux[0, 0] == pytest.approx(1 / 3, abs=1e-12) and r.flux[1, 0] == pytest.approx(-1 / 3, abs=1e-12)
    plan = fg.Plan(two_circuit())
    r = plan.solve([[2.0, 0.0], [0.0, -3.0], [2.0, -3.0], [2.0, np.nan]])
    assert r.status == [0, 0, 0, fg.capi.INVALID_ARGUMENT]
    assert r.a[0, 4] == pytest.approx(0.5, abs=1e-12)
    assert r.a[1, 4] == pytest.approx(-0.375, abs=1e-12)
    assert r.a[2, 4] == pytest.approx(0.125, abs=1e-12)
    np.testing.assert_allclose(r.flux[2], [0.125, 0.0625], atol=1e-12)
    # zero Newton budget -> NONLINEAR_SOLVE_NOT_CONVERGED with zero iterations
    r = plan.solve([[2.0, 0.0]], options=fg.production_options(max_newton_iterations=0))
    assert r.status == [fg.capi.NONLINEAR_SOLVE_NOT_CONVERGED] and r.info[0].iterations == 0


def test_determinism_and_warm_start(gpu):
    model = meshes.square_nonlinear(m=20, seed=8)
    currents = meshes.seeded_currents(4, 3, 20.0, seed=1)
    plan = fg.Plan(model)
    r1 = plan.solve(currents)
    r2 = plan.solve(currents)
    for f in ("a", "b1", "b2", "flux"):
        assert np.array_equal(getattr(r1, f), getattr(r2, f))
    assert [i.iterations for i in r1.info] == [i.iterations for i in r2.info]
    # warm start from the converged field: Newton from iteration 0, no extra steps, same answer
    w = plan.solve(currents, warm=r1.a)
    assert all(s == 0 for s in w.status)
    for k in range(4):
        assert w.info[k].iterations <= r1.info[k].iterations
        assert rel(w.a[k], r1.a[k]) <= 1e-9
    check_solve(model, currents, warm=r1.a)


@pytest.mark.parametrize("k", [1, 5, 16, 32])
def test_batch_widths_match_oracle(gpu, k):
    model = meshes.square_nonlinear(m=14, seed=3)
    check_solve(model, meshes.seeded_currents(k, 3, 20.0, seed=k))


def test_batches_beyond_32_are_chunked(gpu, monkeypatch):
    """A batch of 40: chunks of 32 and 8.  Solved chunk after chunk (the default), its first
    32 items equal a batch of those 32 bit for bit; with the chunks advancing together
    (FG_CHUNKS_TOGETHER=2), within 5e-9 (a chunk then runs on fewer CTAs and its reductions
    round differently) with the same Newton iteration counts."""
    model = meshes.square_nonlinear(m=10, seed=6)
    currents = meshes.seeded_currents(40, 3, 20.0, seed=2)
    plan = fg.Plan(model)
    first = plan.solve(currents[:32])
    monkeypatch.setenv("FG_CHUNKS_TOGETHER", "0")
    r = plan.solve(currents)
    assert all(s == 0 for s in r.status)
    assert np.array_equal(first.a, r.a[:32])
    monkeypatch.setenv("FG_CHUNKS_TOGETHER", "2")
    together = plan.solve(currents)
    assert all(s == 0 for s in together.status)
    for i in range(40):
        assert together.info[i].iterations == r.info[i].iterations
        assert rel(together.a[i], r.a[i]) <= 5e-9


# ----------------------------------------------------------------------------- full size
def test_full_size_linear_superposition(gpu):
    """Linear workload (4,225 nodes): A(I1) + A(I2) = A(I1 + I2) and it matches the oracle."""
    model = meshes.square_linear(m=64)
    plan, got = check_solve(model, np.array([[10.0], [-4.0], [6.0]]))
    assert rel(got.a[0] + got.a[1], got.a[2]) <= 1e-9
    assert rel(got.flux[0] + got.flux[1], got.flux[2]) <= 1e-9


def test_full_size_nonlinear_equation_residual(gpu):
    """250k-node nonlinear workload: converged, and the Newton system at the returned state
    reproduces the state (relative equation residual at the level of the step gate)."""
    model = meshes.square_nonlinear(m=500, seed=2)
    currents = meshes.seeded_currents(2, 3, 20.0, seed=7)
    plan = fg.Plan(model)
    r = plan.solve(currents)
    assert all(s == 0 for s in r.status)
    for k in range(2):
        assert r.info[k].residual_l2 < 1e-6
        assert np.all(np.isfinite(r.flux[k]))
    ro, col, n2f, sign, bnd = plan.symbolic()
    free = np.flatnonzero(n2f >= 0)
    vals, diag, rhs = plan.assemble(r.a, currents, 1)
    for k in range(2):
        x = np.zeros(plan.rows)
        x[n2f[free]] = sign[free] * r.a[k, free]
        rows = np.repeat(np.arange(plan.rows), np.diff(ro))
        Ax = np.bincount(rows, weights=vals[k] * x[col], minlength=plan.rows)
        assert np.linalg.norm(Ax - rhs[k]) <= 1e-5 * np.linalg.norm(rhs[k])


# ----------------------------------------------------------------------------- mixed precision
def check_mixed(model, currents, tol_a=2e-8, tol_flux=1e-8):
    """FP32 inner PCG in FP64 defect correction against the FP64 oracle: same statuses,
    A within tol_a and flux linkage within tol_flux (relative 2-norm).  Both meet the same
    1e-10 true-residual gate along different Krylov paths, so A differs by up to about
    cond(K) x 1e-10 (measured 6e-9 on the 251k-node workload); flux stays within 3e-10."""
    plan = fg.Plan(model, precision=1)
    got = plan.solve(currents)
    a, b1, b2, flux, info = O.solve_batch(model, currents)
    errs = []
    for k in range(len(info)):
        assert got.info[k].status == info[k].status == 0, (got.info[k].status, info[k].status)
        errs.append((rel(got.a[k], a[k]), rel(got.flux[k], flux[k])))
        assert errs[-1][0] <= tol_a and errs[-1][1] <= tol_flux, errs[-1]
    return plan, got, errs


def test_mixed_precision_matches_fp64_oracle(gpu):
    model = meshes.square_nonlinear(m=32, seed=4)
    plan, got, errs = check_mixed(model, meshes.seeded_currents(4, 3, 20.0, seed=9))
    assert plan.last_timing().mixed_fallbacks == 0


def test_mixed_precision_fixtures_and_axisymmetric(gpu):
    model, currents = artifact.read_artifact(open(os.path.join(GOLDEN, "periodic_strip.gpu.json")).read())
    check_mixed(model, currents[None, :])
    check_mixed(meshes.axisymmetric_plunger(mr=12, mz=24), meshes.seeded_currents(2, 2, 30.0, 5))


@pytest.mark.parametrize("form", [dict(precision=1),
                                  dict(precision=1, preconditioner=1, block_size=8, from_iterate=True),
                                  dict(preconditioner=1, block_size=8, from_iterate=True)],
                         ids=["mixed_jacobi", "mixed_block8_from_iterate", "fp64_block8_from_iterate"])
def test_fast_forms_on_the_saturated_sector_match_the_oracle(gpu, form):
    """The accelerated forms on the rotor-stator sector (anti-periodic edges, iron driven to
    2 T, about 30 relaxed Newton iterations) against the FP64 oracle of the plain method:
    same status, Newton iterations within 2, flux linkage within 1e-8 (the bound the
    accelerated forms are held to), A within 5e-8 (different Krylov paths to the same 1e-10
    gate, carried through the relaxed iteration)."""
    model = meshes.annular_sector(nr=24, nt=36)
    currents = np.random.default_rng(41).uniform(-15.0, 15.0, size=(3, 3))
    got = fg.Plan(model, **form).solve(currents)
    a, b1, b2, flux, info = O.solve_batch(model, currents)
    for k in range(3):
        assert got.info[k].status == info[k].status == 0
        assert abs(got.info[k].iterations - info[k].iterations) <= 2
        assert rel(got.flux[k], flux[k]) <= 1e-8, rel(got.flux[k], flux[k])
        assert rel(got.a[k], a[k]) <= 5e-8, rel(got.a[k], a[k])


def test_autotuned_launch_shapes_leave_results_bitwise_unchanged(gpu, monkeypatch):
    """The plan's launch-shape autotuner (fg_plan_pcg_shapes) times the value ring and the
    column cache on the system it is about to solve and keeps the fastest; neither knob
    changes any arithmetic, so a tuned plan answers bit for bit as an untuned one, and the
    timing runs leave no trace in the solve."""
    model = meshes.square_nonlinear(m=60, seed=3)
    currents = meshes.seeded_currents(8, 3, 20.0, seed=13)
    tuned = fg.Plan(model)
    r1 = tuned.solve(currents)
    shapes = tuned.pcg_shapes()
    # 3,481 rows in 28 row groups of 16 warp-steps: an even count, so the 1024-thread CTAs
    # are the fifth candidate
    assert len(shapes) == 1 and shapes[0]["items"] == 8 and shapes[0]["candidates"] == 5
    assert all(t > 0 for t in shapes[0]["us_per_iteration"])
    assert shapes[0]["threads_per_block"] in (512, 1024)
    monkeypatch.setenv("FG_PCG_TUNE", "0")
    plain = fg.Plan(model)
    r2 = plain.solve(currents)
    assert plain.pcg_shapes() == []
    for f in ("a", "b1", "b2", "flux"):
        assert np.array_equal(getattr(r1, f), getattr(r2, f))
    assert [i.linear_iterations for i in r1.info] == [i.linear_iterations for i in r2.info]


@pytest.mark.parametrize("workload", ["square250_k8", "sector_k32"])
def test_wide_ctas_give_the_same_bits(gpu, monkeypatch, workload):
    """CTAs of 1024 threads (two row groups each, one CTA per SM) run the same rows in the
    same per-warp order and store one partial sum per row group, so they answer bit for bit
    as the 512-thread CTAs; the autotuner may therefore pick either shape."""
    if workload == "square250_k8":
        model, currents = meshes.square_nonlinear(m=250, seed=2), meshes.seeded_currents(8, 3, 20.0, seed=7)
    else:
        model = meshes.annular_sector()
        currents = np.random.default_rng(5).uniform(-15.0, 15.0, size=(32, 3))
    monkeypatch.setenv("FG_PCG_TUNE", "0")
    narrow = fg.Plan(model)
    r1 = narrow.solve(currents)
    assert narrow.last_timing().pcg_block == 512
    monkeypatch.setenv("FG_PCG_BLOCK", "1024")
    wide = fg.Plan(model)
    r2 = wide.solve(currents)
    t = wide.last_timing()
    assert t.pcg_block == 1024 and 2 * t.pcg_grid == narrow.last_timing().pcg_grid
    for f in ("a", "b1", "b2", "flux"):
        assert np.array_equal(getattr(r1, f), getattr(r2, f)), f
    assert [i.linear_iterations for i in r1.info] == [i.linear_iterations for i in r2.info]
    monkeypatch.delenv("FG_PCG_BLOCK")
    tuned = fg.Plan(model)
    monkeypatch.delenv("FG_PCG_TUNE")
    r3 = tuned.solve(currents)
    shape = tuned.pcg_shapes()[0]
    assert shape["candidates"] == 5 and shape["us_per_iteration"][4] > 0
    assert np.array_equal(r3.a, r1.a) and np.array_equal(r3.flux, r1.flux)
