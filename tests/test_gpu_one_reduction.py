"""The one-reduction PCG form (FG_PLAN_PCG_ONE_REDUCTION, csrc/pcg1r_kernel.cuh) against the
FP64 oracle of the reference method and against the default two-barrier form.

Chronopoulos and Gear's rearrangement takes both inner products of a CG iteration after
the SpMV, so a launch synchronises its grid once per iteration.  Its rounding differs from
the reference's recurrence, so it is held to the solve's tolerances, not to bits:
* same status and Newton iteration count as the oracle (the reference's driver,
  nonlinear_solver.cu:183-530, on the reference's Jacobi PCG, pcg_kernels.cu:10-344);
* flux linkage within 1e-8 and A within 1e-8 relative 2-norm (two Krylov paths meeting
  the same 1e-10 true-residual gate);
* PCG iterations within 10 % of the default form's;
* a solve repeated on the same plan is bitwise identical;
* an exhausted iteration budget gives the same statuses as the default form, and a grid
  wait that runs out ends the launch with INTERNAL_ERROR on a context that stays usable.
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def check(model, currents, tol_a=1e-8, tol_flux=1e-8):
    plan = fg.Plan(model, one_reduction=True)
    got = plan.solve(currents)
    a, b1, b2, flux, info = O.solve_batch(model, currents)
    for k in range(len(info)):
        assert got.info[k].status == info[k].status == 0, (k, got.info[k].status, info[k].status)
        assert got.info[k].iterations == info[k].iterations, (k, got.info[k].iterations, info[k].iterations)
        assert rel(got.flux[k], flux[k]) <= tol_flux, (k, rel(got.flux[k], flux[k]))
        assert rel(got.a[k], a[k]) <= tol_a, (k, rel(got.a[k], a[k]))
    return plan, got


@pytest.mark.parametrize("k", [1, 5, 32])
def test_one_reduction_matches_oracle_on_the_nonlinear_square(gpu, k):
    model = meshes.square_nonlinear(m=40, seed=6)
    currents = meshes.seeded_currents(k, 3, 20.0, seed=100 + k)
    plan, got = check(model, currents)
    base = fg.Plan(model).solve(currents)
    ours = np.array([i.linear_iterations for i in got.info], float)
    theirs = np.array([i.linear_iterations for i in base.info], float)
    assert np.all(np.abs(ours - theirs) <= 0.1 * theirs + 2), (ours, theirs)
    again = plan.solve(currents)
    for f in ("a", "b1", "b2", "flux"):
        assert np.array_equal(getattr(again, f), getattr(got, f))


def test_one_reduction_on_the_saturated_sector(gpu):
    """The rotor-stator sector: anti-periodic edges, iron driven to 2 T, about 30 relaxed
    Newton iterations of about a thousand PCG iterations each."""
    model = meshes.annular_sector(nr=24, nt=36)
    currents = np.random.default_rng(41).uniform(-15.0, 15.0, size=(3, 3))
    check(model, currents, tol_a=5e-8)


def test_one_reduction_axisymmetric_and_linear(gpu):
    check(meshes.axisymmetric_plunger(mr=12, mz=24), meshes.seeded_currents(2, 2, 30.0, 5))
    check(meshes.square_linear(m=24), np.array([[10.0], [-3.0], [6.0]]))


def test_one_reduction_budget_and_wait_statuses(gpu):
    model = meshes.square_nonlinear(m=30, seed=2)
    currents = meshes.seeded_currents(4, 3, 20.0, seed=17)
    opts = fg.production_options(max_linear_iterations=5, adaptive_linear_tolerance=0)
    one = fg.Plan(model, one_reduction=True).solve(currents, options=opts)
    two = fg.Plan(model).solve(currents, options=opts)
    assert one.status == two.status and all(s != 0 for s in one.status), (one.status, two.status)
    plan = fg.Plan(model, one_reduction=True)
    previous = fg.capi.set_wait_limit_ns(1)
    try:
        with pytest.raises(fg.FgError) as err:
            plan.solve(currents)
        assert err.value.status == fg.capi.INTERNAL_ERROR
    finally:
        assert fg.capi.set_wait_limit_ns(previous) == 1
    assert plan.solve(currents).status == [0] * 4
