"""The oracle and the library's host B-H code against the reference's golden vectors.

Golden data: tests/golden/ (copied from FEMM-GPU gpu_solver/tests/fixtures/35PN230_v1,
see tests/golden/make_golden.py); known answers from gpu_solver/src/bh_curve_poc.cu:
355-380 and gpu_solver/tests/native/physics_regression.cu:45-68.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN
import femm_gpu_b200 as fg


def load_35pn230():
    tab = np.loadtxt(os.path.join(GOLDEN, "35PN230.tab"), skiprows=1)
    return tab[:, 1].copy(), tab[:, 0].copy()  # B, H


def test_35pn230_spline_matches_reference_fixture():
    B, H = load_35pn230()
    assert B.size == 29
    b, h, s, cold, passes = O.bh_build(B, H)
    assert passes == 0
    assert cold == pytest.approx(172.803, rel=0, abs=1e-12)
    # bh_curve_poc.cu:361-362
    assert s[0] == pytest.approx(201.99906442618772, rel=1e-12)
    assert s[-1] == pytest.approx(793566.95194043161, rel=1e-12)
    samples = np.loadtxt(os.path.join(GOLDEN, "35PN230_reference_samples.txt"))
    assert samples.shape == (59, 5)  # 29 knots, 28 midpoints, extrapolation, -B
    for row in samples:
        got = O.bh_eval(b, h, s, row[0])
        for g, e in zip(got, row[1:]):
            assert abs(g - e) <= 1e-12 * max(1.0, abs(e)), (row[0], got, row[1:])


def test_library_host_spline_is_bitwise_the_oracle_and_the_reference():
    B, H = load_35pn230()
    ob, oh, os_, ocold, _ = O.bh_build(B, H)
    pb, ph, ps, pcold, _ = fg.bh_build(B, H)
    assert np.array_equal(os_, ps) and ocold == pcold
    if O.ref() is not None:
        rb, rh, rs, rcold, _ = O.bh_build(B, H, use_ref=True)
        assert np.array_equal(rs, ps) and rcold == pcold
    samples = np.loadtxt(os.path.join(GOLDEN, "35PN230_reference_samples.txt"))
    for row in samples:
        assert np.array_equal(fg.bh_eval(pb, ph, ps, row[0]), O.bh_eval(ob, oh, os_, row[0]))


def test_smoothing_reference():
    ref = np.loadtxt(os.path.join(GOLDEN, "35PN230_smoothing_reference.txt"), skiprows=2)
    passes_expected = int(open(os.path.join(GOLDEN, "35PN230_smoothing_reference.txt")).read().split("\n")[1])
    for build in (O.bh_build, fg.bh_build):
        b, h, s, cold, passes = build([0.0, 1.0, 2.0, 3.0], [0.0, 1.0, 1.01, 10.0])
        assert passes == passes_expected == 1
        # rows: B_T H_A_per_m dH_dB after smoothing
        np.testing.assert_allclose(b, ref[:, 0], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(h, ref[:, 1], rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(s, ref[:, 2], rtol=1e-13, atol=1e-14)
        assert cold == 1.0  # first secant of the raw curve


def test_analytic_spline_and_extrapolation():
    # bh_curve_poc.cu:365-380: natural spline slopes of (0,0), (1,1), (2,4).
    for build, ev in ((O.bh_build, O.bh_eval), (fg.bh_build, fg.bh_eval)):
        b, h, s, _, _ = build([0.0, 1.0, 2.0], [0.0, 1.0, 4.0])
        np.testing.assert_allclose(s, [0.5, 2.0, 3.5], rtol=1e-15)
        # linear extrapolation beyond the last knot with the last slope
        out = ev(b, h, s, 3.0)
        assert out[0] == pytest.approx(4.0 + 3.5)
        assert out[1] == pytest.approx(3.5, rel=1e-14)
        # B = 0 returns the initial slope as reluctivity
        out = ev(b, h, s, 0.0)
        assert out[2] == 0.5 and out[3] == 0.0
        # negative B is symmetric
        np.testing.assert_array_equal(ev(b, h, s, -1.3), ev(b, h, s, 1.3))


def test_invalid_curves_rejected():
    for build in (O.bh_build, fg.bh_build):
        with pytest.raises(ValueError):
            build([0.0, 1.0, 1.0], [0.0, 1.0, 2.0])  # not strictly increasing
        with pytest.raises(ValueError):
            build([0.1, 1.0], [0.0, 1.0])  # does not start at the origin
