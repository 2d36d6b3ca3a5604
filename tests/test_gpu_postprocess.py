"""GPU tests of the frozen postprocess: the mask solved by the library's PCG, force /
torque / air-gap B on GPU solutions, the device form, and the CLI paths that serve them.

Tolerances:
* --single-sample against FEMM 4.2's frozen values: the reference's own gates
  (FrozenPostprocessReferenceTest, gpu_solver/tests/native/reference_commands.cu:175-195):
  |d| <= abs + rel |FEMM| with Fx / Fy 1e-8 + 1e-5, torque 1e-10 + 1e-5, radial B
  1e-9 + 1e-5, flux linkage 1e-10 + 1e-6;
* the mask: equal to the reference's (0 / 1 per node, no tolerance);
* the library's host postprocess of a GPU solution: equal bit for bit to the reference's
  ComputeFrozenPostprocess on the same solution and mask;
* the device form against the host form: radial B to 1e-13 relative of the largest sample
  (the same operations in the same order with explicit rounding, except that FEMM's
  sharp-corner fallback takes |B| from the device hypot, which may differ from the host's
  in the last bits); force and torque to 1e-12 relative of the largest partial magnitude
  (per-CTA partial sums instead of one sequential sum).
"""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from conftest import GOLDEN, ROOT
from femm_gpu_b200 import artifact, meshes
from test_postprocess_host import (STEM, describe_femm, element_b, frozen_reference, model_from_description,
                                   paired_mask_model, sector_model)

pytestmark = pytest.mark.gpu
CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


def near(got, want, absolute, relative):
    return np.isfinite(got) and abs(got - want) <= absolute + relative * abs(want)


def single_sample_request(tmp_path):
    req = json.load(open(os.path.join(GOLDEN, "nonlinear_pm_coil_single_sample_request.json")))
    req["stem"], req["curve_directory"] = STEM, GOLDEN
    p = tmp_path / "single.json"
    p.write_text(json.dumps(req, indent=2))
    return p, req


def test_single_sample_matches_femm_within_reference_gates(gpu, tmp_path):
    rq, req = single_sample_request(tmp_path)
    rs = tmp_path / "resp.json"
    r = subprocess.run([CLI, "--single-sample", str(rq), str(rs)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    body = json.loads(rs.read_text())
    fx, fy, tq, _, deg, radial = frozen_reference()
    assert body["status"] == "PASS" and body["solve_status"] == "PASS" and body["error_identifier"] == ""
    assert body["source_motor_fem_sha256"] == req["source_motor_fem_sha256"]
    assert near(body["Fx_N"], fx, 1e-8, 1e-5) and near(body["Fy_N"], fy, 1e-8, 1e-5), body
    assert near(body["torque_Nm"], tq, 1e-10, 1e-5), body
    flux = json.load(open(os.path.join(GOLDEN, "expected.json")))["nonlinear_pm_coil_planar"]["flux_linkage_Wb"]
    assert near(body["circuit_flux_linkage_Wb"][0], flux, 1e-10, 1e-6)
    assert body["actual_circuit_currents_A"] == [5.0] and body["mesh_element_count"] == 890
    assert body["airgap_sample_angles_deg"] == list(deg)
    for got, want in zip(body["airgap_radial_flux_density_T"], radial):
        assert near(got, want, 1e-9, 1e-5), (got, want)
    assert body["convergence"]["iterations"] > 0


@needs_ref
def test_gpu_mask_and_postprocess_equal_the_reference(gpu):
    h, _, _, _ = O.ref_femm_nonlinear(STEM, GOLDEN)
    model = model_from_description(describe_femm()[1])
    _, _, _, radius, deg, _ = frozen_reference()
    ang = deg * np.pi / 180.0
    plan = fg.Plan(model)
    sol = plan.solve([[5.0]], options=fg.capi.FgSolveOptions(1e-8, 128, 128, 1e-13, 0, 0))
    assert sol.info[0].status == 0
    pp = fg.Postprocess(plan, radius_m=radius, angles_rad=ang)
    st, fx, fy, tq, radial, ref_mask = O.ref_postprocess(h, sol.a[0], sol.b1[0], sol.b2[0], radius_m=radius,
                                                         angles_rad=ang)
    assert st == 0 and np.array_equal(pp.mask(), ref_mask)
    r = pp.compute(sol.a, sol.b1, sol.b2)
    assert r.status[0] == 0
    assert r.force[0, 0] == fx and r.force[0, 1] == fy and r.torque[0] == tq
    assert np.array_equal(r.radial_b[0], radial)


@needs_ref
def test_periodic_sector_mask_on_gpu_equals_reference(gpu):
    sec = sector_model(nr=96, nt=150)
    hs = O.ref_model_handle(sec)
    plan = fg.Plan(sec)
    pp = fg.Postprocess(plan, selected_group=10, air_group=0, radius_m=0.0455,
                        angles_rad=np.radians(np.linspace(1.0, 89.0, 45)), max_mask_iterations=4096)
    zeros_n, zeros_e = np.zeros(sec.node_count), np.zeros(sec.tri_count)
    st, *_, ref_mask = O.ref_postprocess(hs, zeros_n, zeros_e, zeros_e, selected_group=10, air_group=0,
                                         max_mask_iterations=4096)
    assert st == 0 and np.array_equal(pp.mask(), ref_mask)
    assert np.array_equal(O.weighted_stress_mask(sec, 10, 0, by_group=True), ref_mask)


@needs_ref
def test_gpu_mask_with_apex_node_and_antiperiodic_pair_equals_reference(gpu):
    """physics_regression.cu:225-251: the apex node's Dirichlet zero is no mask boundary and
    the anti-periodic pair is tied with sign +1; without the apex entry both refuse alike."""
    model, apex = paired_mask_model()
    z_n, z_e = np.zeros(model.node_count), np.zeros(model.tri_count)
    st, *_, ref_mask = O.ref_postprocess(O.ref_model_handle(model, apex_nodes=apex), z_n, z_e, z_e,
                                         selected_label=1, air_label=0)
    assert st == 0
    plan = fg.Plan(model)
    pp = fg.Postprocess(plan, selected_label=1, air_label=0, apex_nodes=apex)
    got = pp.mask()
    assert np.array_equal(got, ref_mask) and got[6] == got[8] and got[12] == 1.0
    st_plain, *_ = O.ref_postprocess(O.ref_model_handle(model), z_n, z_e, z_e, selected_label=1, air_label=0)
    with pytest.raises(fg.FgError) as e:
        fg.Postprocess(plan, selected_label=1, air_label=0)
    assert st_plain != 0 and e.value.status == st_plain


def test_device_postprocess_matches_host_form(gpu):
    import torch
    sec = sector_model(nr=96, nt=150)
    plan = fg.Plan(sec)
    currents = meshes.seeded_currents(6, 3, 8.0, seed=4)
    sol = plan.solve(currents)
    assert all(i.status == 0 for i in sol.info)
    pp = fg.Postprocess(plan, selected_group=10, air_group=0, radius_m=0.0455,
                        angles_rad=np.radians(np.linspace(1.0, 89.0, 45)), max_mask_iterations=4096)
    host = pp.compute(sol.a, sol.b1, sol.b2)
    dev = [torch.from_numpy(x).cuda().contiguous() for x in (sol.a, sol.b1, sol.b2)]
    torch.cuda.synchronize()
    got = pp.compute_device(6, dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr())
    assert (got.status == 0).all() and (host.status == 0).all()
    scale_b = np.abs(host.radial_b).max()
    np.testing.assert_allclose(got.radial_b, host.radial_b, rtol=0, atol=1e-13 * scale_b)
    scale = np.abs(host.force).max() + np.abs(host.torque).max() / 0.05
    np.testing.assert_allclose(got.force, host.force, rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(got.torque, host.torque, rtol=0, atol=1e-12 * scale * 0.05)
    # the rotor torque of a magnet sector is not zero
    assert np.abs(host.torque).min() > 0


def legacy_artifact(tmp_path):
    """A planar-DC artifact with one block-label group per region (no node constraints)."""
    text, _ = artifact.write_artifact(meshes.square_linear(m=12), [12.0])
    src = json.loads(text)
    src["schema_version"] = "gpu_femm_planar_dc_mesh_v1"
    res = src["resolved"]
    del res["node_constraints"]
    for i, r in enumerate(res["regions"]):
        r["group_number"] = i
    src["canonical_identity_sha256"] = artifact.canonical_sha256(artifact._loads(json.dumps(src))["resolved"])
    path = tmp_path / "legacy.gpu.json"
    path.write_text(json.dumps(src))
    return path, sorted({int(r["group_number"]) for r in res["regions"]})


def sample(path, currents, **kw):
    r = {"protocol": "gpu_femm_planar_dc_sample_v1", "mesh_artifact_path": str(path),
         "mesh_artifact_sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(),
         "circuit_currents_A": list(map(float, currents)), "force_group_number": -1,
         "stress_air_group_number": -1, "airgap_radius_mm": 0, "airgap_angles_deg": [],
         "sliding_band_angle_deg": 0, "compute_force_torque": False, "include_field_solution": False}
    r.update(kw)
    return r


def call(tmp_path, command, body):
    rq, rs = tmp_path / "in.json", tmp_path / "out.json"
    rq.write_text(json.dumps(body))
    r = subprocess.run([CLI, command, str(rq), str(rs)], capture_output=True, text=True, timeout=600)
    return r.returncode, json.loads(rs.read_text()), r.stderr


@needs_ref
def test_cli_solve_serves_force_and_torque_like_the_reference(gpu, tmp_path):
    path, groups = legacy_artifact(tmp_path)
    h = O.ref_artifact_handle(open(path, "rb").read())
    model, _ = O._ref_model(h.h)
    # (2, 0) is served; (1, 0) fixes a node to both 1 and 0 (BOUNDARY_INVALID) and (0, 1)
    # selects a region touching another non-air region (INVALID_MATERIAL).
    assert groups == [0, 1, 2, 3]
    for sel, air in ((2, 0), (1, 0), (0, 1)):
        req = sample(path, [12.0], compute_force_torque=True, force_group_number=sel,
                     stress_air_group_number=air, include_field_solution=True)
        rc, body, err = call(tmp_path, "--solve", req)
        ref_st = O.ref_postprocess(h, np.zeros(model.node_count), np.zeros(model.tri_count),
                                   np.zeros(model.tri_count), selected_group=sel, air_group=air,
                                   max_mask_iterations=4096)[0]
        if ref_st != 0:
            assert rc == 1 and body["solve_status"] == "OK"
            assert body["postprocess_status"] == fg.status_name(ref_st) and body["Fx_N"] is None
            continue
        assert rc == 0, err
        assert body["status"] == "PASS" and body["postprocess_status"] == "OK"
        a = np.array(body["node_A_Wb_per_m"])
        b1, b2 = np.array(body["element_Bx_T"]), np.array(body["element_By_T"])
        st, fx, fy, tq, _, _ = O.ref_postprocess(h, a, b1, b2, selected_group=sel, air_group=air,
                                                 max_mask_iterations=4096)
        assert st == 0
        assert body["Fx_N"] == fx and body["Fy_N"] == fy and body["torque_Nm"] == tq
        assert body["airgap_sample_angles_deg"] == [] and body["airgap_radial_flux_density_T"] == []


def test_cli_batch_shares_the_mask_and_matches_single_solves(gpu, tmp_path):
    path, groups = legacy_artifact(tmp_path)
    items = []
    for i, cur in enumerate((12.0, -4.0, 7.5, 0.5)):
        items.append({"task_id": f"t{i}", "request": sample(path, [cur], compute_force_torque=True,
                                                           force_group_number=2, stress_air_group_number=0)})
    batch = {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 4, "items": items}
    rc, body, err = call(tmp_path, "--batch", batch)
    single = [call(tmp_path, "--solve", it["request"])[1] for it in items]
    assert {s["postprocess_status"] for s in single} == {"OK"} and body["status"] == "PASS"
    for it, one in zip(body["items"], single):
        resp = it["response"]
        assert resp["postprocess_status"] == one["postprocess_status"]
        if one["postprocess_status"] != "OK":
            continue
        assert resp["status"] == "PASS"
        for key in ("Fx_N", "Fy_N", "torque_Nm"):
            assert abs(resp[key] - one[key]) <= 1e-8 * max(abs(one[key]), 1e-12), key
