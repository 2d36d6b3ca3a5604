"""The frozen postprocess (weighted-stress force / torque, smoothed air-gap B) on the CPU.

Pins, in order:

* the reference's own ComputeFrozenPostprocess (oracle/_ref: field_postprocess.cpp and
  weighted_stress.cu compiled here, the mask's device solve replaced by the oracle's CPU
  PCG), fed FEMM 4.2's nodal A from the nonlinear PM / coil fixture, reproduces FEMM's
  frozen weighted-stress force, torque and mo_getb air-gap samples
  (nonlinear_pm_coil_planar.postprocess.txt) to 1e-12;
* the numpy mask restatement (oracle.weighted_stress_mask) equals the reference's mask;
* the product's FEMM .ans reader (femm_gpu --describe-femm-ans) builds the reference
  reader's model bit for bit;
* the product's host postprocess (fg_postprocess_compute on a host-only plan, mask given)
  equals the reference bit for bit, and its plan statuses follow the reference's.

The GPU mask solve and the device postprocess are checked in test_gpu_postprocess.py.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from conftest import GOLDEN, ROOT
from femm_gpu_b200 import meshes

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
STEM = os.path.join(GOLDEN, "nonlinear_pm_coil_planar")
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


def frozen_reference():
    """FEMM's frozen values: (Fx, Fy, torque, radius_m, angles_deg, radial_b)."""
    kv, angles, radial = {}, [], []
    for line in open(STEM + ".postprocess.txt"):
        line = line.strip()
        if line.startswith("airgap_sample_deg="):
            fields = dict(f.split("=") for f in line.split())
            angles.append(float(fields["airgap_sample_deg"]))
            radial.append(float(fields["radial_B_T"]))
        elif "=" in line:
            k, v = line.split("=", 1)
            kv[k] = v
    return (float(kv["Fx_N"]), float(kv["Fy_N"]), float(kv["torque_Nm"]),
            float(kv["airgap_radius_mm"]) * 1e-3, np.array(angles), np.array(radial))


def element_b(model, a):
    """Element B from nodal A, as the reference computes it (sum over corners of A b_x, A b_y)."""
    p = model.xy[model.tri]
    det = ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1])
           - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    dx = np.stack([p[:, 1, 1] - p[:, 2, 1], p[:, 2, 1] - p[:, 0, 1], p[:, 0, 1] - p[:, 1, 1]], 1)
    dy = np.stack([p[:, 2, 0] - p[:, 1, 0], p[:, 0, 0] - p[:, 2, 0], p[:, 1, 0] - p[:, 0, 0]], 1)
    bx, by = dy / det[:, None], -dx / det[:, None]
    av = a[model.tri]
    b1 = ((0.0 + av[:, 0] * bx[:, 0]) + av[:, 1] * bx[:, 1]) + av[:, 2] * bx[:, 2]
    b2 = ((0.0 + av[:, 0] * by[:, 0]) + av[:, 1] * by[:, 1]) + av[:, 2] * by[:, 2]
    return b1, b2


def describe_femm(stem=STEM, curves=GOLDEN):
    r = subprocess.run([CLI, "--describe-femm-ans", stem, curves], capture_output=True, text=True, timeout=60)
    return r.returncode, json.loads(r.stdout)


def model_from_description(d):
    mats = np.array(d["materials"])
    return fg.Model(
        xy=np.array(d["xy"]).reshape(-1, 2), tri=np.array(d["tri"]).reshape(-1, 3), tri_mat=d["tri_mat"],
        nu0=mats[:, 0], alpha=mats[:, 1], j_per_a=mats[:, 2], hc=mats[:, 3], mag_deg=mats[:, 4],
        curve_index=mats[:, 5].astype(int), circuit_index=mats[:, 6].astype(int),
        group=mats[:, 7].astype(int), curves=[(np.array(b), np.array(h)) for b, h in d["curves"]],
        dir_nodes=d["dirichlet_nodes"], dir_values=np.zeros(len(d["dirichlet_nodes"])),
        circuit_count=len(d["circuit_currents_A"]), depth_m=d["depth_m"], problem_type=d["problem_type"])


@needs_ref
def test_reference_postprocess_reproduces_femm_from_femm_solution():
    h, model, a, _ = O.ref_femm_nonlinear(STEM, GOLDEN)
    fx, fy, tq, radius, deg, radial = frozen_reference()
    b1, b2 = element_b(model, a)
    st, gx, gy, gt, grad, mask = O.ref_postprocess(h, a, b1, b2, radius_m=radius, angles_rad=deg * np.pi / 180.0)
    assert st == 0
    for got, want in ((gx, fx), (gy, fy), (gt, tq)):
        assert abs(got - want) <= 1e-12 * abs(want), (got, want)
    np.testing.assert_allclose(grad, radial, rtol=1e-12, atol=1e-15)
    assert set(np.unique(mask)) == {0.0, 1.0}


@needs_ref
def test_numpy_mask_restatement_equals_reference_mask():
    h, model, a, _ = O.ref_femm_nonlinear(STEM, GOLDEN)
    b1, b2 = element_b(model, a)
    st, *_, mask = O.ref_postprocess(h, a, b1, b2)
    assert st == 0 and np.array_equal(O.weighted_stress_mask(model, 1, 3), mask)
    # a periodic sector: rotor iron + magnets as one group against the air group
    sec = sector_model()
    hs = O.ref_model_handle(sec)
    zeros = np.zeros(sec.node_count)
    st, *_, mask = O.ref_postprocess(hs, zeros, np.zeros(sec.tri_count), np.zeros(sec.tri_count),
                                     selected_group=10, air_group=0)
    assert st == 0
    assert np.array_equal(O.weighted_stress_mask(sec, 10, 0, by_group=True), mask)
    assert 0 < mask.sum() < sec.node_count


def paired_mask_model():
    """The reference's paired-mask case (tests/native/physics_regression.cu:225-251 on
    LargeStructuredMaskFixture(4), tests/native/fixtures.cpp:47-84): a 5 x 5 node grid, 1 m
    cells, the selected label 1 on the one triangle (12, 13, 18), label 0 elsewhere (the
    air), the outer ring held at 0, an anti-periodic pair 6 ~ 8 and node 12 Dirichlet too.
    Returns (model, apex_nodes)."""
    side = 5
    xy = np.array([(x, y) for y in range(side) for x in range(side)], np.float64)
    tri, mat = [], []
    for y in range(side - 1):
        for x in range(side - 1):
            ll = y * side + x
            lr, ul = ll + 1, ll + side
            ur = ul + 1
            tri += [(ll, lr, ur), (ll, ur, ul)]
            mat += [1 if ll == 12 else 0, 0]
    ring = [y * side + x for y in range(side) for x in range(side)
            if x in (0, side - 1) or y in (0, side - 1)]
    dirichlet = ring + [12]
    nu = 1.0 / meshes.MU0
    model = fg.Model(xy=xy, tri=tri, tri_mat=mat, nu0=[nu, nu], alpha=[0.0, 0.0], j_per_a=[0.0, 0.0],
                     hc=[0.0, 0.0], mag_deg=[0.0, 0.0], curve_index=[-1, -1], circuit_index=[-1, -1],
                     group=[0, 1], curves=[], dir_nodes=dirichlet, dir_values=np.zeros(len(dirichlet)),
                     con_a=[6], con_b=[8], con_sign=[-1], circuit_count=1)
    return model, [12]


@needs_ref
def test_mask_ignores_apex_zero_and_ties_periodic_pairs_like_the_reference():
    model, apex = paired_mask_model()
    st, *_, mask = O.ref_postprocess(O.ref_model_handle(model, apex_nodes=apex), np.zeros(25), np.zeros(32),
                                     np.zeros(32), selected_label=1, air_label=0)
    assert st == 0 and mask[6] == mask[8] and mask[12] == 1.0
    assert np.array_equal(O.weighted_stress_mask(model, 1, 0, apex_nodes=apex), mask)
    # without the apex entry node 12 is both Dirichlet 0 and selected 1: the reference refuses
    st_plain, *_ = O.ref_postprocess(O.ref_model_handle(model), np.zeros(25), np.zeros(32), np.zeros(32),
                                     selected_label=1, air_label=0)
    assert st_plain != 0 and O.weighted_stress_mask(model, 1, 0) is None
    with pytest.raises(fg.FgError) as e:  # refused before any GPU work
        fg.Postprocess(fg.Plan(model, host_only=True), selected_label=1, air_label=0)
    assert e.value.status == st_plain


def sector_model(nr=48, nt=72):
    m = meshes.annular_sector(nr=nr, nt=nt)
    m.group = np.array([0, 10, 10, 3, 4, 5, 6], np.int32)
    return m


@needs_ref
def test_femm_reader_builds_the_reference_model():
    rc, d = describe_femm()
    assert rc == 0 and d["plan_status"] == "OK"
    h, ref_model, _, _ = O.ref_femm_nonlinear(STEM, GOLDEN)
    ours = model_from_description(d)
    assert np.array_equal(ours.xy, ref_model.xy) and np.array_equal(ours.tri, ref_model.tri)
    assert np.array_equal(ours.tri_mat, ref_model.tri_mat)
    for f in ("nu0", "alpha", "j_per_a", "hc", "mag_deg", "curve_index", "circuit_index", "group"):
        assert np.array_equal(getattr(ours, f), getattr(ref_model, f)), f
    assert np.array_equal(ours.dir_nodes, ref_model.dir_nodes)
    assert ours.depth_m == ref_model.depth_m == 0.020
    assert np.array_equal(ours.curves[0][0], ref_model.curves[0][0])
    assert np.array_equal(ours.curves[0][1], ref_model.curves[0][1])


def test_femm_reader_errors(tmp_path):
    bad = tmp_path / "bad"
    text = open(STEM + ".ans").read()
    # an out-of-range block label
    lines = text.split("\n")
    k = lines.index("[Solution]")
    n = int(lines[k + 1])
    first_element = k + 2 + n + 1
    parts = lines[first_element].split()
    parts[3] = "7"
    lines[first_element] = " ".join(parts)
    (tmp_path / "bad.ans").write_text("\n".join(lines))
    rc, d = describe_femm(str(bad))
    assert rc == 1 and d["error"] == "missing or out-of-range nonlinear block label"
    rc, d = describe_femm(str(tmp_path / "missing"))
    assert rc == 1 and d["error"] == "invalid nonlinear [Solution] node count"
    rc, d = describe_femm(STEM, str(tmp_path))
    assert rc == 1 and d["error"] == "cannot read 35PN230 B-H table"


@needs_ref
def test_host_postprocess_is_the_reference_bit_for_bit():
    h, model, a, _ = O.ref_femm_nonlinear(STEM, GOLDEN)
    _, fy, _, radius, deg, _ = frozen_reference()
    b1, b2 = element_b(model, a)
    ang = deg * np.pi / 180.0
    st, fx, fy, tq, radial, mask = O.ref_postprocess(h, a, b1, b2, radius_m=radius, angles_rad=ang)
    plan = fg.Plan(model_from_description(describe_femm()[1]), host_only=True)
    pp = fg.Postprocess(plan, radius_m=radius, angles_rad=ang, mask=mask)
    assert pp.probes == 4 and np.array_equal(pp.mask(), mask)
    r = pp.compute(a, b1, b2)
    assert r.status[0] == 0
    assert r.force[0, 0] == fx and r.force[0, 1] == fy and r.torque[0] == tq
    assert np.array_equal(r.radial_b[0], radial)
    # several items at once, each its own answer
    rng = np.random.default_rng(3)
    aa = np.stack([a, a * 0.5, a + 1e-4 * rng.standard_normal(a.size)])
    bb = [element_b(model, x) for x in aa]
    rk = pp.compute(aa, np.stack([b[0] for b in bb]), np.stack([b[1] for b in bb]))
    for i in range(3):
        st, fx, fy, tq, radial, _ = O.ref_postprocess(h, aa[i], bb[i][0], bb[i][1], radius_m=radius,
                                                      angles_rad=ang, mask=mask)
        assert rk.status[i] == 0 and rk.force[i, 0] == fx and rk.force[i, 1] == fy and rk.torque[i] == tq
        assert np.array_equal(rk.radial_b[i], radial)


@needs_ref
def test_sector_host_postprocess_bit_exact_with_smoothing_at_interfaces():
    """Probes in the air gap and between magnets: corners on label interfaces take FEMM's
    interface traversal (Bt from the source side, Bn from A)."""
    sec = sector_model()
    hs = O.ref_model_handle(sec)
    rng = np.random.default_rng(11)
    a = 1e-2 * rng.standard_normal(sec.node_count)
    a[sec.dir_nodes] = 0.0
    b1, b2 = element_b(sec, a)
    _, *_, mask = O.ref_postprocess(hs, a, b1, b2, selected_group=10, air_group=0)
    for radius, deg in ((0.0455, np.linspace(1.0, 89.0, 17)), (0.044, np.array([5.0, 10.0, 80.0])),
                        (0.04501, np.array([30.0, 47.3]))):
        ang = np.radians(deg)
        st, fx, fy, tq, radial, _ = O.ref_postprocess(hs, a, b1, b2, selected_group=10, air_group=0,
                                                      radius_m=radius, angles_rad=ang, mask=mask)
        assert st == 0
        pp = fg.Postprocess(fg.Plan(sec, host_only=True), selected_group=10, air_group=0, radius_m=radius,
                            angles_rad=ang, mask=mask)
        r = pp.compute(a, b1, b2)
        assert r.status[0] == 0 and r.force[0, 0] == fx and r.force[0, 1] == fy and r.torque[0] == tq
        assert np.array_equal(r.radial_b[0], radial)


@needs_ref
def test_plan_statuses_follow_the_reference():
    """Mask-building refusals (checked before any GPU work) and probe refusals (with the
    mask given, BuildFrozenPostprocessPlanWithMask) carry the reference's status."""
    h, model, a, _ = O.ref_femm_nonlinear(STEM, GOLDEN)
    b1, b2 = element_b(model, a)
    plan = fg.Plan(model_from_description(describe_femm()[1]), host_only=True)
    _, *_, mask = O.ref_postprocess(h, a, b1, b2)

    def ref_status(kw, with_mask):
        ref_kw = dict(kw)
        for k, v in (("selected_label", 1), ("air_label", 3), ("selected_group", -1), ("air_group", -1)):
            ref_kw.setdefault(k, v)
        return O.ref_postprocess(h, a, b1, b2, mask=mask if with_mask else None, **ref_kw)[0]

    mask_cases = [
        dict(selected_label=7),                    # label out of range
        dict(selected_label=3, air_label=3),       # selected == air
        dict(selected_label=1, air_label=2),       # the magnet touches other air: refused by MakeMask
        dict(selected_group=2, air_group=2),       # equal groups
        dict(selected_group=5, air_group=6),       # absent group: nothing selected
        dict(max_mask_iterations=0),
        dict(mask_tolerance=0.0),
    ]
    probe_cases = [
        dict(radius_m=1.0, angles_rad=[0.0]),      # probe outside the mesh
        dict(radius_m=6e-3, angles_rad=[0.0]),     # probe inside the magnet, not air
        dict(radius_m=1e-3, angles_rad=[np.nan]),  # non-finite angle
        dict(radius_m=-1.0),
    ]
    for kw, with_mask in [(c, False) for c in mask_cases] + [(c, True) for c in probe_cases]:
        st = ref_status(kw, with_mask)
        assert st != 0, kw
        with pytest.raises(fg.FgError) as e:
            fg.Postprocess(plan, mask=mask if with_mask else None, **kw)
        assert e.value.status == st, (kw, e.value.status, st)


def test_postprocess_refuses_axisymmetric_plans_and_bad_masks():
    axi = meshes.axisymmetric_plunger(mr=8, mz=16)
    with pytest.raises(fg.FgError) as e:
        fg.Postprocess(fg.Plan(axi, host_only=True), mask=np.zeros(axi.node_count))
    assert e.value.status == fg.capi.UNSUPPORTED_FEATURE
    sq = meshes.square_linear(m=8)
    plan = fg.Plan(sq, host_only=True)
    with pytest.raises(fg.FgError) as e:
        fg.Postprocess(plan, selected_label=0, air_label=1, mask=np.full(sq.node_count, 0.5))
    assert e.value.status == fg.capi.INVALID_ARGUMENT


def test_device_postprocess_refuses_without_gpu_on_host_only_plan():
    sq = meshes.square_linear(m=8)
    plan = fg.Plan(sq, host_only=True)
    pp = fg.Postprocess(plan, selected_label=0, air_label=1, mask=np.zeros(sq.node_count))
    with pytest.raises(fg.FgError) as e:
        pp.compute_device(1, 0, 0, 0)
    assert e.value.status in (fg.capi.GPU_UNAVAILABLE, fg.capi.INVALID_ARGUMENT)
