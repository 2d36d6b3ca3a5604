"""CPU oracle against the reference's frozen stock-FEMM answers and known-answer tests.

* periodic_strip_v1 / antiperiodic_strip_v1: flux linkage within 1e-10 relative of stock
  FEMM (the reference's own gate, test_femm_gpu_cli.py:223-283); every constraint pair
  equal or negated;
* axisymmetric_coil_v1: flux within 1e-3 (P1 vs FEMM's r^2 basis, :286-293);
* unit-square and two-circuit known answers (gpu_solver/tests/native/self_test.cu:139-199,
  :261-294, fixtures.cpp:6-16, :105-120);
* the Python artifact reader matches the reference's strict parser field by field.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN
from femm_gpu_b200 import artifact
from femm_gpu_b200.model import Model

EXPECTED = json.load(open(os.path.join(GOLDEN, "expected.json")))


def load(name):
    text = open(os.path.join(GOLDEN, name + ".gpu.json")).read()
    return artifact.read_artifact(text)


@pytest.mark.parametrize("name,rtol", [("periodic_strip", 1e-10), ("antiperiodic_strip", 1e-10),
                                       ("axisymmetric_coil", 1e-3)])
def test_oracle_flux_matches_stock_femm(name, rtol):
    model, currents = load(name)
    a, b1, b2, flux, info = O.solve_batch(model, currents[None, :])
    assert info[0].status == 0
    expected = EXPECTED[name]["flux_linkage_Wb"]
    assert abs(flux[0, 0] - expected) <= rtol * abs(expected)
    if model.con_a.size:
        pair = a[0, model.con_b] - model.con_sign * a[0, model.con_a]
        assert np.max(np.abs(pair)) <= 1e-15 * np.max(np.abs(a))


@pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["periodic_strip", "antiperiodic_strip", "axisymmetric_coil"])
def test_artifact_reader_matches_reference_parser(name):
    R = O.ref()
    text = open(os.path.join(GOLDEN, name + ".gpu.json"), "rb").read()
    h = C.c_void_p()
    assert R.ref_parse_artifact(text, C.c_size_t(len(text)), C.byref(h)) == 0
    sizes = np.zeros(8, np.int32)
    depth, ptype = C.c_double(), C.c_int32()
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    R.ref_artifact_sizes(h, p(sizes), C.byref(depth), C.byref(ptype))
    N, E, M = sizes[:3]
    xy, tri, tm = np.zeros(2 * N), np.zeros(3 * E, np.int32), np.zeros(E, np.int32)
    md, mi = np.zeros(5 * M), np.zeros(3 * M, np.int32)
    cb = np.zeros(max(sizes[7], 1))
    ch, cs = np.zeros_like(cb), np.zeros_like(cb)
    dn = np.zeros(sizes[4], np.int32)
    con = np.zeros(3 * max(sizes[5], 1), np.int32)
    cu = np.zeros(max(sizes[6], 1))
    R.ref_artifact_copy(h, p(xy), p(tri), p(tm), p(md), p(mi), p(cb), p(ch), p(cs), p(dn), p(con), p(cu))
    R.ref_artifact_free(h)
    model, currents = artifact.read_artifact(text.decode())
    md = md.reshape(M, 5)
    mi = mi.reshape(M, 3)
    assert np.array_equal(xy.reshape(-1, 2), model.xy)
    assert np.array_equal(tri.reshape(-1, 3), model.tri) and np.array_equal(tm, model.tri_mat)
    for col, field in enumerate(("nu0", "alpha", "j_per_a", "hc", "mag_deg")):
        assert np.array_equal(md[:, col], getattr(model, field)), field
    assert np.array_equal(mi[:, 0], model.curve_index) and np.array_equal(mi[:, 1], model.circuit_index)
    assert np.array_equal(dn, model.dir_nodes)
    c3 = con[: 3 * sizes[5]].reshape(-1, 3)
    assert np.array_equal(c3[:, 0], model.con_a) and np.array_equal(c3[:, 1], model.con_b)
    assert np.array_equal(c3[:, 2], model.con_sign)
    assert depth.value == model.depth_m and ptype.value == model.problem_type
    assert np.array_equal(cu[: sizes[6]], currents)


def unit_square(jpa=1.0):
    """fixtures.cpp:6-16 as a nonlinear-path model: nu = 1, J = 1 per amp on all four triangles."""
    return Model(xy=[[0, 0], [1, 0], [1, 1], [0, 1], [0.5, 0.5]],
                 tri=[[0, 1, 4], [1, 2, 4], [2, 3, 4], [3, 0, 4]], tri_mat=[0, 0, 0, 0],
                 nu0=[1.0], alpha=[0.0], j_per_a=[jpa], hc=[0.0], mag_deg=[0.0], curve_index=[-1],
                 circuit_index=[0], group=[0], curves=[], dir_nodes=[0, 1, 2, 3],
                 dir_values=[0, 0, 0, 0], circuit_count=1, depth_m=1.0, name="unit_square")


def two_circuit():
    """NonlinearTwoCircuitFixture (fixtures.cpp:105-120)."""
    return Model(xy=[[0, 0], [1, 0], [1, 1], [0, 1], [0.5, 0.5]],
                 tri=[[0, 1, 4], [1, 2, 4], [2, 3, 4], [3, 0, 4]], tri_mat=[1, 0, 2, 0],
                 nu0=[1.0, 1.0, 1.0], alpha=[0, 0, 0], j_per_a=[0.0, 12.0, 6.0], hc=[0, 0, 0],
                 mag_deg=[0, 0, 0], curve_index=[-1, -1, -1], circuit_index=[-1, 0, 1],
                 group=[0, 1, 2], curves=[], dir_nodes=[0, 1, 2, 3], dir_values=[0, 0, 0, 0],
                 circuit_count=2, depth_m=1.0, name="two_circuit")


def test_unit_square_known_answer():
    a, b1, b2, flux, info = O.solve_batch(unit_square(), np.array([[12.0], [-12.0]]))
    assert [i.status for i in info] == [0, 0]
    np.testing.assert_allclose(a[0], [0, 0, 0, 0, 1.0], atol=1e-12)
    np.testing.assert_allclose(b1[0], [2.0, 0.0, -2.0, 0.0], atol=1e-12)
    np.testing.assert_allclose(b2[0], [0.0, 2.0, 0.0, -2.0], atol=1e-12)
    assert flux[0, 0] == pytest.approx(1.0 / 3.0, abs=1e-12)
    np.testing.assert_allclose(a[1], -a[0], atol=1e-12)
    assert flux[1, 0] == pytest.approx(-1.0 / 3.0, abs=1e-12)


def test_two_circuit_superposition():
    a, b1, b2, flux, info = O.solve_batch(two_circuit(), np.array([[2.0, 0.0], [0.0, -3.0], [2.0, -3.0]]))
    assert all(i.status == 0 for i in info)
    assert a[0, 4] == pytest.approx(0.5, abs=1e-12)
    assert a[1, 4] == pytest.approx(-0.375, abs=1e-12)
    assert a[2, 4] == pytest.approx(0.125, abs=1e-12)
    np.testing.assert_allclose(flux[2], [0.125, 0.0625], atol=1e-12)


def test_nonfinite_current_isolated_in_batch():
    a, b1, b2, flux, info = O.solve_batch(two_circuit(), np.array([[2.0, np.nan], [2.0, -3.0]]))
    assert info[0].status == 2 and info[1].status == 0
    assert a[1, 4] == pytest.approx(0.125, abs=1e-12)
