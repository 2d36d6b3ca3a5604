"""FEMM's native air-gap element (AGE) on the CPU: the element matrix, the host plan's
fixed band terms and validation, against the reference's own code (oracle/_ref compiles
native_airgap_matrix.cpp with its matrix body cut from FEMM's fkn/prob1big.cpp, as the
reference's build does, and its PrepareNonlinearAssembly / ValidateNonlinearModel).

Tolerances:
* element matrix: the library derives it as T^T Q T (Catmull-Rom corner interpolation,
  four-corner form) instead of FEMM's expanded polynomials, so the two agree to rounding:
  |d| <= 1e-13 max|ref| over random band terms;
* symbolic CSR with the band couples, free-row maps and the triangle contributors:
  bit-exact;
* the band stiffness per CSR slot and the fixed-node load: |d| <= 1e-13 max|ref|;
* validation statuses: equal.
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes

REF = O.ref()
needs_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref not built (no reference checkout)")


def close(got, want, scale_tol=1e-13):
    want = np.asarray(want)
    return np.max(np.abs(np.asarray(got) - want)) <= scale_tol * max(np.max(np.abs(want)), 1e-300)


@needs_ref
def test_element_matrix_restatement_equals_femm_matrix():
    rng = np.random.default_rng(3)
    cases = [(0.75, 0.25, 0.75), (1.0, 1.0, 1.0), (0.3, 1.0, 0.0), (2.5, 1e-9, 1.0), (0.05, 0.5, 0.0)]
    cases += [(rng.uniform(0.02, 4.0), rng.uniform(0, 1), float(rng.integers(0, 2))) for _ in range(40)]
    cases += [(rng.uniform(0.02, 4.0), rng.uniform(0, 1), rng.uniform(0, 1)) for _ in range(40)]
    for K, ci, co in cases:
        ref = O.ref_age_matrix(K, 1.0 / K, ci, co)
        mine = O.age_matrix(K, 1.0 / K, ci, co)
        assert close(mine, ref), (K, ci, co)
        # symmetric, constants in the null space, rank 3 (a four-corner element)
        assert np.allclose(mine, mine.T, rtol=0, atol=1e-15 * np.abs(mine).max())
        assert np.abs(mine.sum(axis=1)).max() <= 1e-14 * np.abs(mine).max()
        assert np.linalg.matrix_rank(mine, tol=1e-10 * np.abs(mine).max()) == 3
    for bad in ((0.0, 1.0, 0.5, 0.5), (1.0, -1.0, 0.5, 0.5), (np.inf, 1.0, 0.5, 0.5), (1.0, 1.0, np.nan, 0.5)):
        assert O.ref_age_matrix(*bad) is None


def band_models():
    yield meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=0.0)
    yield meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=7.3)
    # fixed ring nodes with non-zero values: the band loads the free rows next to them
    m = meshes.sliding_band_machine(nr=40, nt=24, rotor_deg=2.0)
    ring = m.ages[0].nodes[:6, 1]
    m.dir_nodes = np.concatenate([m.dir_nodes, ring]).astype(np.int32)
    m.dir_values = np.concatenate([m.dir_values, np.linspace(1e-3, -2e-3, ring.size)])
    m.name = "sliding_band_fixed_ring"
    yield m
    # an anti-periodic band closure (weights carry the copy signs)
    m = meshes.sliding_band_machine(nr=40, nt=24, rotor_deg=4.0)
    g = m.ages[0]
    g.antiperiodic = True
    g.weights[: g.weights.shape[0] // 2] *= -1.0
    m.name = "sliding_band_antiperiodic_records"
    yield m


@needs_ref
@pytest.mark.parametrize("model", list(band_models()), ids=lambda m: m.name)
def test_band_pattern_and_fixed_terms_match_reference(model):
    from test_host_topology import PAIR, ref_prepared
    plan = fg.Plan(model, host_only=True)
    ro, col, *_ = plan.symbolic()
    ref = ref_prepared(model)
    assert np.array_equal(ro, ref["ro"]) and np.array_equal(col, ref["col"])
    so, se, rro, re, pm, cr = plan.contributors()
    assert np.array_equal(so, ref["moff"]) and np.array_equal(rro, ref["roff"])
    assert np.array_equal(se[:, 1], PAIR[ref["ment"][:, 1], ref["ment"][:, 2]])
    assert np.array_equal(re, ref["rent"]) and np.array_equal(pm, ref["pm"])
    st, ref_val, ref_rhs = O.ref_prepared_age(model)
    assert st == 0
    val, rhs = plan.air_gap()
    assert close(val, ref_val)
    assert np.array_equal(val == 0.0, ref_val == 0.0)
    if np.any(ref_rhs != 0.0):
        assert close(rhs, ref_rhs)
    else:
        assert not np.any(rhs)


@needs_ref
def test_models_without_a_band_report_zero_band_terms():
    plan = fg.Plan(meshes.square_linear(m=6), host_only=True)
    val, rhs = plan.air_gap()
    assert not val.any() and not rhs.any()


@needs_ref
def test_band_validation_statuses_match_reference():
    def variant(edit):
        m = meshes.sliding_band_machine(nr=40, nt=12)
        edit(m, m.ages[0])
        return m

    def short(m, g):
        g.nodes, g.weights = g.nodes[:2].copy(), g.weights[:2].copy()

    def node_out(m, g):
        g.nodes[3, 2] = m.node_count

    def weight_nan(m, g):
        g.weights[1, 0] = np.nan

    def radii(m, g):
        g.outer_radius_m = g.inner_radius_m

    def arc(m, g):
        g.arc_length_deg = 0.0

    def shift(m, g):
        g.inner_shift = np.inf

    def inner_zero(m, g):
        g.inner_radius_m = 0.0

    cases = [short, node_out, weight_nan, radii, arc, shift, inner_zero]
    for edit in cases:
        m = variant(edit)
        want = O.validate(m, use_ref=True)
        assert want == fg.capi.MESH_INVALID, edit.__name__
        with pytest.raises(fg.FgError) as err:
            fg.Plan(m, host_only=True)
        assert err.value.status == want, edit.__name__
    # a band on an axisymmetric model is refused as unsupported
    axi = meshes.axisymmetric_plunger(mr=6, mz=8)
    axi.ages = [fg.AirGap(nodes=np.zeros((4, 4), np.int32), weights=np.ones((4, 4)), inner_radius_m=0.01,
                          outer_radius_m=0.02, arc_length_deg=360.0)]
    assert O.validate(axi, use_ref=True) == fg.capi.UNSUPPORTED_FEATURE
    with pytest.raises(fg.FgError) as err:
        fg.Plan(axi, host_only=True)
    assert err.value.status == fg.capi.UNSUPPORTED_FEATURE


@needs_ref
def test_band_stands_in_for_the_meshed_gap():
    """Physics check of the synthetic sliding-band machine through the reference's own CPU
    Newton path: at rotor angle 0 the band model and the machine with its gap meshed give the
    same flux linkage to 1e-3, and turning the rotor changes it."""
    cur = np.array([[8.0, -4.0, -4.0]])
    _, flux_mesh, st, *_ = O.ref_cpu_newton_batch(meshes.two_pole_machine(nr=40, nt=30, full=True), cur)
    _, flux_band, st2, *_ = O.ref_cpu_newton_batch(meshes.sliding_band_machine(nr=40, nt=30), cur)
    assert st[0] == 0 and st2[0] == 0
    assert np.abs(flux_band - flux_mesh).max() <= 1e-3 * np.abs(flux_mesh).max()
    _, flux_turned, st3, *_ = O.ref_cpu_newton_batch(meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=30.0),
                                                     cur)
    assert st3[0] == 0 and np.abs(flux_turned - flux_band).max() > 0.1 * np.abs(flux_band).max()


def test_restatement_refuses_band_models():
    """The plain-C restatement carries no air-gap element: it refuses such models instead of
    assembling them without the band (band models are checked against oracle/_ref)."""
    assert O.validate(meshes.sliding_band_machine(nr=40, nt=12)) == fg.capi.UNSUPPORTED_FEATURE
