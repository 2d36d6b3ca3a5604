"""GPU parity of the native air-gap element (AGE) path: sliding-band machines solved by
libfemmgpu (through the C ABI) against the reference's own host code in oracle/_ref (its
AssembleNonlinearNewton and its CPU Newton path with FEMM's PCG, both carrying the band).

Tolerances:
* assembly: the reference's NearMixed(1e-12, 5e-11) host / device gate
  (protocol_contract_tests.cu:963-1013), the absolute part scaled to the system's magnitude;
  repeated assembly bitwise identical;
* Newton solves at relative tolerance 1e-11 and linear tolerance 1e-13 on both sides: every
  item converges; flux linkage within 1e-8 and A within 1e-7 (relative 2-norms) of the
  reference CPU path, whose own production-to-tight drift on these models is 4e-9 (flux)
  and 8e-8 (A).
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@needs_ref
@pytest.mark.parametrize("deg", [0.0, 7.3])
def test_band_assembly_matches_reference(gpu, deg):
    model = meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=deg)
    plan = fg.Plan(model)
    ro, col, *_ = plan.symbolic()
    rng = np.random.default_rng(11)
    states = rng.normal(size=(3, model.node_count)) * 3e-3
    states[:, model.dir_nodes] = 0.0
    currents = rng.uniform(-15, 15, size=(3, model.circuit_count))
    for use_newton in (0, 1):
        vals, diag, rhs = plan.assemble(states, currents, use_newton)
        for k in range(3):
            ref = O.assemble(model, states[k], currents[k], use_newton, use_ref=True)
            assert np.array_equal(ro, ref.off) and np.array_equal(col, ref.col)
            for got, exp in ((vals[k], ref.val), (diag[k], ref.diag), (rhs[k], ref.rhs)):
                tol = 1e-12 * np.max(np.abs(exp)) + 5e-11 * np.abs(exp)
                assert np.all(np.abs(got - exp) <= tol), np.max(np.abs(got - exp) / (np.abs(exp) + 1e-300))
        again = plan.assemble(states, currents, use_newton)
        for x, y in zip((vals, diag, rhs), again):
            assert np.array_equal(x, y)


@needs_ref
@pytest.mark.parametrize("deg", [0.0, 7.3, 33.0])
def test_band_newton_solves_match_reference_cpu_path(gpu, deg):
    model = meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=deg)
    currents = meshes.seeded_currents(3, 3, 10.0, seed=2)
    tight = O.production_options(relative_tolerance=1e-11, linear_relative_tolerance=1e-13)
    a, flux, status, *_ = O.ref_cpu_newton_batch(model, currents, options=tight, threads=3)
    assert (status == 0).all()
    plan = fg.Plan(model)
    opts = fg.production_options()
    opts.relative_tolerance, opts.linear_relative_tolerance = 1e-11, 1e-13
    got = plan.solve(currents, options=opts)
    for k in range(currents.shape[0]):
        assert got.info[k].status == 0
        assert rel(got.flux[k], flux[k]) <= 1e-8, rel(got.flux[k], flux[k])
        assert rel(got.a[k], a[k]) <= 1e-7, rel(got.a[k], a[k])


@needs_ref
def test_band_solve_through_block_jacobi_and_mixed_forms(gpu):
    """The accelerated forms serve band models too: same converged answer to the forms'
    own acceptance (flux within 1e-8 of the plain FP64 method)."""
    model = meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=12.0)
    currents = meshes.seeded_currents(2, 3, 10.0, seed=5)
    base = fg.Plan(model).solve(currents)
    assert all(i.status == 0 for i in base.info)
    for plan in (fg.Plan(model, preconditioner=1, block_size=8), fg.Plan(model, precision=1)):
        got = plan.solve(currents)
        for k in range(2):
            assert got.info[k].status == 0
            assert rel(got.flux[k], base.flux[k]) <= 1e-8
