"""Tangent multi-RHS at a converged field (SolveTangentMultiRhs, nonlinear_solver.cu:85-172)
and its postprocess (ComputeFrozenTangentPostprocess, field_postprocess.cpp:405-520) on the
CPU.

* The oracle's restatement of the tangent solve passes the reference's own check
  (protocol_contract_tests.cu:194-264): central differences of nonlinear solves at h and
  h/2 approach the tangent dA, the h/2 error below the h error and below 5e-4, with the
  linear residual below 1e-10.
* The reference's tangent postprocess is the bilinear cross term: 0.5 (F(B + dB) -
  F(B - dB)) to 1e-12 (protocol_contract_tests.cu:265-300).
* The product's host tangent postprocess (fg_postprocess_tangent, host-only plan, mask
  given) equals the reference's bit for bit.
The GPU tangent solve is checked against this oracle in test_gpu_tangent.py.
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes
from test_postprocess_host import element_b, sector_model

needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), np.finfo(float).tiny)


def solved(model, currents):
    a, b1, b2, flux, info = O.solve_batch(model, np.atleast_2d(currents))
    assert info[0].status == 0
    return a[0], b1[0], b2[0], flux[0]


def nonlinear_model():
    """The reference check's set-up: every material nu = nu0 (1 + 0.3 |B|^2)."""
    model = meshes.square_nonlinear(m=20, seed=3)
    model.alpha[:] = 0.3
    model.curve_index[:] = -1
    return model


BASE = np.array([600.0, -400.0, 300.0])


def test_oracle_tangent_matches_central_differences():
    model = nonlinear_model()
    base = BASE[: model.circuit_count]
    a0, *_ = solved(model, base)
    dirs = np.eye(model.circuit_count)[:2]
    da, db1, db2, dflux, infos = O.tangent(model, a0, base, dirs)
    for st, its, res in infos:
        assert st == 0 and res < 1e-10
    for i in range(2):
        def central(h):
            plus, minus = base.copy(), base.copy()
            plus[i] += h
            minus[i] -= h
            ap, *_ = solved(model, plus)
            am, *_ = solved(model, minus)
            return (ap - am) / (2 * h)
        e_h, e_h2 = rel(central(20.0), da[i]), rel(central(10.0), da[i])
        assert e_h2 < e_h and e_h2 < 5e-4, (e_h, e_h2)
        # flux derivatives are the linear evaluation of dA
        _, _, fl = O.finalize(model, da[i])
        np.testing.assert_array_equal(fl, dflux[i])


@needs_ref
def test_reference_tangent_postprocess_is_the_bilinear_cross_term():
    sec = sector_model()
    hs = O.ref_model_handle(sec)
    rng = np.random.default_rng(5)
    a = 1e-2 * rng.standard_normal(sec.node_count)
    da = 1e-4 * rng.standard_normal(sec.node_count)
    a[sec.dir_nodes] = 0.0
    da[sec.dir_nodes] = 0.0
    b1, b2 = element_b(sec, a)
    db1, db2 = element_b(sec, da)
    _, *_, mask = O.ref_postprocess(hs, a, b1, b2, selected_group=10, air_group=0)
    ang = np.radians([10.0, 45.0, 80.0])
    kw = dict(selected_group=10, air_group=0, radius_m=0.0455, angles_rad=ang)
    st, dfx, dfy, dtq, drad = O.ref_tangent_postprocess(hs, a, b1, b2, da, db1, db2, mask, **kw)
    assert st == 0
    plus = O.ref_postprocess(hs, a + da, b1 + db1, b2 + db2, mask=mask, **kw)
    minus = O.ref_postprocess(hs, a - da, b1 - db1, b2 - db2, mask=mask, **kw)
    for k, got in ((1, dfx), (2, dfy), (3, dtq)):
        want = 0.5 * (plus[k] - minus[k])
        assert abs(got - want) <= 1e-12 + 1e-12 * abs(want), (k, got, want)
    # the air-gap derivative is the smoothing of dA, dB alone
    lin = O.ref_postprocess(hs, da, db1, db2, mask=mask, **kw)
    np.testing.assert_array_equal(drad, lin[4])

    # the product's host tangent postprocess: the reference bit for bit
    plan = fg.Plan(sec, host_only=True)
    pp = fg.Postprocess(plan, selected_group=10, air_group=0, radius_m=0.0455, angles_rad=ang, mask=mask)
    r = pp.tangent(b1, b2, np.stack([da, 2 * da]), np.stack([db1, 2 * db1]), np.stack([db2, 2 * db2]))
    assert (r.status == 0).all()
    assert r.force[0, 0] == dfx and r.force[0, 1] == dfy and r.torque[0] == dtq
    assert np.array_equal(r.radial_b[0], drad)
    st2 = O.ref_tangent_postprocess(hs, a, b1, b2, 2 * da, 2 * db1, 2 * db2, mask, **kw)
    assert r.force[1, 0] == st2[1] and r.force[1, 1] == st2[2] and r.torque[1] == st2[3]
    assert np.array_equal(r.radial_b[1], st2[4])


def test_tangent_refuses_without_gpu_and_validates():
    model = meshes.square_nonlinear(m=8, seed=1)
    plan = fg.Plan(model, host_only=True)
    with pytest.raises(fg.FgError) as e:
        plan.solve_tangent(np.zeros(model.node_count), np.zeros(model.circuit_count), np.eye(model.circuit_count))
    assert e.value.status == fg.capi.GPU_UNAVAILABLE
