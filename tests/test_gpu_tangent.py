"""GPU tests of the tangent multi-RHS (fg_solve_tangent) and its postprocess.

Tolerances: dA, dB and dflux against the oracle's restatement within 1e-9 relative (both
PCGs stop at the relative residual 1e-13; the Jacobian's condition number turns that into
about 1e-10 on the solution); linearity in the directions within 1e-9; the central-
difference check of the reference (h/2 error below the h error and below 5e-4); the
tangent postprocess of a GPU tangent equal bit for bit to the reference's on the same
inputs.
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes
from test_postprocess_host import sector_model
from test_tangent_host import BASE, nonlinear_model, rel

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
TIGHT = dict(linear_relative_tolerance=1e-13, max_linear_iterations=4096)


def options(**kw):
    o = fg.production_options()
    for k, v in {**TIGHT, **kw}.items():
        setattr(o, k, v)
    return o


@pytest.mark.parametrize("pre", [(0, 8), (1, 8), (1, 32)])
def test_tangent_matches_oracle(gpu, pre):
    model = nonlinear_model()
    base = BASE[: model.circuit_count]
    plan = fg.Plan(model, preconditioner=pre[0], block_size=pre[1])
    sol = plan.solve([base])
    assert sol.info[0].status == 0
    dirs = np.vstack([np.eye(model.circuit_count), [[0.5, -1.0, 2.0][: model.circuit_count]]])
    da, db1, db2, dflux, info = plan.solve_tangent(sol.a[0], base, dirs, options())
    oa, ob1, ob2, of, oinfo = O.tangent(model, sol.a[0], base, dirs)
    for i in range(dirs.shape[0]):
        assert info[i].status == 0 and info[i].residual_l2 < 1e-10, (i, info[i].status)
        assert rel(da[i], oa[i]) < 1e-9 and rel(db1[i], ob1[i]) < 1e-9 and rel(db2[i], ob2[i]) < 1e-9
        np.testing.assert_allclose(dflux[i], of[i], rtol=1e-9, atol=1e-9 * np.abs(of).max())
    assert np.all(da[:, model.dir_nodes] == 0.0)
    # symmetric differential inductance matrix (reciprocity of the consistent Jacobian)
    L = dflux[: model.circuit_count]
    np.testing.assert_allclose(L, L.T, rtol=1e-8, atol=1e-10 * np.abs(L).max())


def test_tangent_matches_central_differences_on_gpu(gpu):
    model = nonlinear_model()
    base = BASE[: model.circuit_count]
    plan = fg.Plan(model)
    o = fg.production_options()
    a0 = plan.solve([base], options=o).a[0]
    da, *_ = plan.solve_tangent(a0, base, np.eye(model.circuit_count)[:1], options())

    def central(h):
        plus, minus = base.copy(), base.copy()
        plus[0] += h
        minus[0] -= h
        r = plan.solve([plus, minus], options=o)
        assert all(i.status == 0 for i in r.info)
        return (r.a[0] - r.a[1]) / (2 * h)
    e_h, e_h2 = rel(central(20.0), da[0]), rel(central(10.0), da[0])
    assert e_h2 < e_h and e_h2 < 5e-4, (e_h, e_h2)


def test_many_directions_are_linear_and_chunked(gpu):
    model = nonlinear_model()
    base = BASE[: model.circuit_count]
    plan = fg.Plan(model)
    a0 = plan.solve([base]).a[0]
    rng = np.random.default_rng(9)
    d = rng.standard_normal((20, model.circuit_count))
    dirs = np.vstack([d, d[:10] + d[10:], 3.0 * d[:10]])  # 40 directions: two launches
    da, db1, db2, dflux, info = plan.solve_tangent(a0, base, dirs, options())
    assert all(i.status == 0 for i in info)
    assert plan.last_timing().pcg_launches == 2
    for j in range(10):
        assert rel(da[20 + j], da[j] + da[10 + j]) < 1e-9
        assert rel(da[30 + j], 3.0 * da[j]) < 1e-9


def test_tangent_argument_errors(gpu):
    model = nonlinear_model()
    base = BASE[: model.circuit_count]
    plan = fg.Plan(model)
    a0 = plan.solve([base]).a[0]
    bad = a0.copy()
    bad[3] = np.nan
    _, _, _, _, info = plan.solve_tangent(bad, base, np.eye(model.circuit_count), options())
    assert all(i.status == fg.capi.INVALID_ARGUMENT for i in info)
    _, _, _, _, info = plan.solve_tangent(a0, base, np.eye(model.circuit_count),
                                          options(linear_relative_tolerance=0.0))
    assert all(i.status == fg.capi.INVALID_ARGUMENT for i in info)


@needs_ref
def test_sector_torque_derivative_equals_reference(gpu):
    sec = sector_model(nr=96, nt=150)
    hs = O.ref_model_handle(sec)
    plan = fg.Plan(sec)
    base = np.array([6.0, -3.0, -3.0])
    sol = plan.solve([base])
    assert sol.info[0].status == 0
    # The reference's motor options (linear tolerance 1e-10): 1e-13 is below the FP64 floor
    # of the saturated sector's Jacobian (the oracle's PCG stalls near 1e-12 as well).
    da, db1, db2, dflux, info = plan.solve_tangent(sol.a[0], base, np.eye(3), fg.production_options())
    assert all(i.status == 0 for i in info), [(i.status, i.iterations, i.residual_l2) for i in info]
    ang = np.radians(np.linspace(2.0, 88.0, 12))
    pp = fg.Postprocess(plan, selected_group=10, air_group=0, radius_m=0.0455, angles_rad=ang,
                        max_mask_iterations=4096)
    mask = pp.mask()
    r = pp.tangent(sol.b1[0], sol.b2[0], da, db1, db2)
    for i in range(3):
        st, dfx, dfy, dtq, drad = O.ref_tangent_postprocess(
            hs, sol.a[0], sol.b1[0], sol.b2[0], da[i], db1[i], db2[i], mask, selected_group=10, air_group=0,
            radius_m=0.0455, angles_rad=ang)
        assert st == 0 and r.status[i] == 0
        assert r.force[i, 0] == dfx and r.force[i, 1] == dfy and r.torque[i] == dtq
        assert np.array_equal(r.radial_b[i], drad)
    assert np.abs(r.torque).max() > 0
