"""GPU tests of the motor adapters on a posed motor artifact (gpu_femm_mesh_v1).

* --motor-single-sample equals --solve's postprocessed planar-DC response of the same mesh
  bit for bit (same solve, same postprocess);
* --motor-batch items equal their single-sample responses within 1e-9 relative (a batch
  runs a wider PCG launch), tangent blocks equal the library's fg_solve_tangent /
  fg_postprocess_tangent on the single-sample base state within 1e-8 and the flux
  derivatives agree with central differences of single-sample solves within 1e-5 (their
  truncation error);
* a motor transaction through --worker answers as --motor-batch-profile does.
"""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import femm_gpu_b200 as fg
from test_gpu_postprocess import legacy_artifact, sample as planar_sample
from test_postprocess_host import model_from_description
from test_worker_cli import envelope, run_worker

pytestmark = pytest.mark.gpu
CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "femm-gpu_b200", "bin", "femm_gpu")
BASE = "e" * 64


def motor_artifact(tmp_path):
    legacy, _ = legacy_artifact(tmp_path)
    src = json.load(open(legacy))
    src["schema_version"] = "gpu_femm_mesh_v1"
    src["base_motor_fem_sha256"] = BASE
    res = src["resolved"]
    res["base_motor_fem_sha256"] = BASE
    res["pose"] = {"rotor_angle_deg": 0, "displacement_mm": [0, 0]}
    path = tmp_path / "motor.gpu.json"
    path.write_text(json.dumps(src))
    return path, legacy, src["source_fem_sha256"]


def motor_request(path, source, currents, protocol="gpu_femm_motor_sample_v1", **kw):
    r = {"protocol": protocol, "mesh_artifact_path": str(path),
         "mesh_artifact_sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(),
         "base_motor_fem_sha256": BASE, "source_fem_sha256": source,
         "circuit_currents_A": [float(c) for c in currents], "selected_group_number": 2, "air_group_number": 0,
         "airgap_radius_mm": 0, "airgap_angles_deg": [], "rotor_angle_deg": 0, "displacement_mm": [0, 0]}
    if protocol == "gpu_femm_motor_sample_v2":
        r["tangent_multi_rhs"] = None
    r.update(kw)
    return r


def call(tmp_path, command, body, name="in.json"):
    rq, rs = tmp_path / name, tmp_path / ("out_" + name)
    rq.write_text(json.dumps(body))
    r = subprocess.run([CLI, command, str(rq), str(rs)], capture_output=True, text=True, timeout=600)
    return r.returncode, json.loads(rs.read_text()), r.stderr


def test_motor_single_sample_equals_solve(gpu, tmp_path):
    path, legacy, source = motor_artifact(tmp_path)
    rc, m, err = call(tmp_path, "--motor-single-sample", motor_request(path, source, [12.0]))
    assert rc == 0 and m["status"] == "PASS", err
    rc2, s, _ = call(tmp_path, "--solve", planar_sample(legacy, [12.0], compute_force_torque=True,
                                                         force_group_number=2, stress_air_group_number=0),
                     name="solve.json")
    assert rc2 == 0
    for key in ("Fx_N", "Fy_N", "torque_Nm", "circuit_flux_linkage_Wb", "convergence"):
        assert m[key] == s[key], key
    assert m["base_motor_fem_sha256"] == BASE and m["mesh_element_count"] == s["mesh_element_count"]


def test_motor_batch_with_tangent(gpu, tmp_path):
    path, _, source = motor_artifact(tmp_path)
    tangent = {"schema_version": "gpu_femm_tangent_multi_rhs_v1",
               "rhs": [{"name": "d", "circuit_current_derivative_A_per_A": [1.0]},
                       {"name": "half", "circuit_current_derivative_A_per_A": [0.5]}]}
    currents = [12.0, -6.0, 3.0]
    items = [(f"t{i}", motor_request(path, source, [c], "gpu_femm_motor_sample_v2", tangent_multi_rhs=tangent))
             for i, c in enumerate(currents)]
    body = {"protocol": "gpu_femm_motor_batch_v2", "max_items_per_chunk": 4,
            "items": [{"task_id": t, "request": r} for t, r in items]}
    rc, b, err = call(tmp_path, "--motor-batch", body, name="batch.json")
    assert rc == 0 and b["status"] == "PASS", err
    assert b["cache"]["actual_parallel_width"] == 3 and b["cache"]["mesh_cache_hits"] == 2
    model = model_from_description(json.loads(subprocess.run([CLI, "--describe-artifact", str(path)],
                                                             capture_output=True, text=True).stdout))
    plan = fg.Plan(model)
    pp = fg.Postprocess(plan, selected_group=2, air_group=0, max_mask_iterations=4096)
    for (t, req), item in zip(items, b["items"]):
        resp = item["response"]
        v1 = {k: v for k, v in req.items() if k != "tangent_multi_rhs"} | {"protocol": "gpu_femm_motor_sample_v1"}
        rc1, one, _ = call(tmp_path, "--motor-single-sample", v1, name=f"{t}.json")
        assert rc1 == 0
        for key in ("Fx_N", "Fy_N", "torque_Nm"):
            assert abs(resp[key] - one[key]) <= 1e-9 * max(abs(one[key]), 1e-12), key
        f, g = resp["circuit_flux_linkage_Wb"][0], one["circuit_flux_linkage_Wb"][0]
        assert abs(f - g) <= 1e-9 * abs(g)
        tb = resp["tangent_multi_rhs"]
        assert tb["status"] == "PASS" and [r["name"] for r in tb["rhs"]] == ["d", "half"]
        # the library on the single-sample base state
        sol = plan.solve([req["circuit_currents_A"]])
        da, db1, db2, dflux, info = plan.solve_tangent(sol.a[0], req["circuit_currents_A"], [[1.0], [0.5]])
        r = pp.tangent(sol.b1[0], sol.b2[0], da, db1, db2)
        for k, rhs in enumerate(tb["rhs"]):
            assert abs(rhs["circuit_flux_linkage_derivative_Wb_per_A"][0] - dflux[k, 0]) <= 1e-8 * abs(dflux[k, 0])
            assert abs(rhs["dtorque_Nm_per_A"] - r.torque[k]) <= 1e-8 * max(abs(r.torque[k]), 1e-12)
            assert rhs["linear_convergence"]["iterations"] > 0
        # the half direction is half the unit one (linearity of the tangent)
        d0, d1 = tb["rhs"][0], tb["rhs"][1]
        assert abs(d1["circuit_flux_linkage_derivative_Wb_per_A"][0] -
                   0.5 * d0["circuit_flux_linkage_derivative_Wb_per_A"][0]) <= 1e-9 * abs(
            d0["circuit_flux_linkage_derivative_Wb_per_A"][0])
        # central differences of single-sample solves
        h = 0.5
        fl = []
        for c in (req["circuit_currents_A"][0] + h, req["circuit_currents_A"][0] - h):
            rc3, o3, _ = call(tmp_path, "--motor-single-sample",
                              {k: v for k, v in req.items() if k != "tangent_multi_rhs"} |
                              {"protocol": "gpu_femm_motor_sample_v1", "circuit_currents_A": [c]}, name="cd.json")
            fl.append(o3["circuit_flux_linkage_Wb"][0])
        cd = (fl[0] - fl[1]) / (2 * h)
        L = d0["circuit_flux_linkage_derivative_Wb_per_A"][0]
        assert abs(L - cd) <= 1e-5 * abs(L), (L, cd)


def test_motor_transaction_in_worker(gpu, tmp_path):
    path, _, source = motor_artifact(tmp_path)
    body = {"protocol": "gpu_femm_motor_batch_v1", "max_items_per_chunk": 2,
            "items": [{"task_id": f"m{i}", "request": motor_request(path, source, [c])}
                      for i, c in enumerate((12.0, 1.0, -3.0))]}
    b = tmp_path / "mb.json"
    b.write_text(json.dumps(body))
    out = tmp_path / "out"
    out.mkdir()
    st = run_worker([envelope(1, b, out / "w.json")])
    assert st[0]["exit_code"] == 0 and st[0]["error"] == ""
    got = json.load(open(out / "w.json"))
    rc, ref, _ = call(tmp_path, "--motor-batch-profile", body, name="p.json")
    assert rc == 0 and "timing" in got and "timing" in ref
    assert [i["response"] for i in got["items"]] == [i["response"] for i in ref["items"]]
    assert got["cache"] == ref["cache"]


def test_sector_batch_reconstructs_the_full_machine(gpu, tmp_path):
    """A v3 sector batch (half of a two-pole machine, antiperiodic; 0.25 mm radial cells so
    that the air gap holds free mask nodes) reports the full
    machine: its torque, flux linkages and air-gap samples equal a solve of the full
    360-degree mesh within 1e-6 (two discretisations of one field that agree up to the
    Newton and PCG tolerances); its force is zero by the orbit rule and the full machine's
    is zero to roundoff.  The tangent block follows the reference's reconstruction rules on
    the library's tangent of the periodic (suspension-order) operator."""
    from femm_gpu_b200 import meshes
    from test_motor_cli import sector_artifact_text
    sector = meshes.two_pole_machine(nr=160, nt=72)
    full = meshes.two_pole_machine(nr=160, nt=72, full=True)
    source = "f" * 64
    path = tmp_path / "sector.gpu.json"
    path.write_text(sector_artifact_text(sector, base=BASE, source=source))
    digest = hashlib.sha256(open(path, "rb").read()).hexdigest()
    angles = [10.0, 100.0, 190.0, 280.0, 350.0]
    tangent = {"schema_version": "gpu_femm_tangent_multi_rhs_v1",
               "rhs": [{"name": "a", "circuit_current_derivative_A_per_A": [1.0, 0.0, 0.0]}]}
    currents = [[6.0, -3.0, -3.0], [0.0, 4.0, -4.0]]
    items = []
    for i, cur in enumerate(currents):
        items.append({"task_id": f"s{i}", "request": {
            "protocol": "gpu_femm_motor_sample_v3", "mesh_artifact_path": str(path), "mesh_artifact_sha256": digest,
            "base_motor_fem_sha256": BASE, "source_fem_sha256": source, "circuit_currents_A": cur,
            "selected_group_number": 20, "air_group_number": 50, "airgap_radius_mm": 45.5,
            "airgap_angles_deg": angles, "rotor_angle_deg": 0, "displacement_mm": [0, 0],
            "tangent_multi_rhs": tangent,
            "sector_performance": {"schema_version": "gpu_femm_motor_sector_performance_v1",
                                   "model_invariance_certificate_sha256": "d" * 64}}})
    body = {"protocol": "gpu_femm_motor_batch_v3", "max_items_per_chunk": 4, "items": items}
    rc, b, err = call(tmp_path, "--motor-batch", body, name="sector.json")
    assert rc == 0 and b["status"] == "PASS", (err, [(i["response"]["solve_status"],
                                                      i["response"]["convergence"]) for i in b["items"]])
    fplan = fg.Plan(full)
    fsol = fplan.solve(currents)
    fpp = fg.Postprocess(fplan, selected_group=20, air_group=50, radius_m=0.0455,
                         angles_rad=np.radians(angles), max_mask_iterations=4096)
    fres = fpp.compute(fsol.a, fsol.b1, fsol.b2)
    # the library's tangent of the suspension-order (periodic) operator at the sector base
    tmodel = meshes.two_pole_machine(nr=160, nt=72)
    tmodel.con_sign[:] = 1
    tplan, splan = fg.Plan(tmodel), fg.Plan(sector)
    spp = fg.Postprocess(splan, selected_group=20, air_group=50, radius_m=0.0455,
                         angles_rad=np.radians([10.0, 100.0, 10.0, 100.0, 170.0]), max_mask_iterations=4096)
    for i, item in enumerate(b["items"]):
        r = item["response"]
        sr = r["sector_reconstruction"]
        assert sr["status"] == "PASS" and sr["base_torque_multiplier"] == 2 and sr["base_field_repeat_sign"] == -1
        assert sr["tangent_field_repeat_sign"] == 1 and sr["tangent_force_multiplier"] == 2
        assert sr["tangent_torque_multiplier"] == 0 and sr["tangent_rhs_count"] == 1
        assert r["Fx_N"] == 0.0 and r["Fy_N"] == 0.0
        scale = max(abs(fres.torque[i]), 1e-9)
        assert abs(r["torque_Nm"] - fres.torque[i]) <= 1e-6 * scale, (r["torque_Nm"], fres.torque[i])
        assert np.abs(fres.force[i]).max() <= 1e-6 * max(1.0, np.abs(fres.torque[i]) / 0.05)
        np.testing.assert_allclose(r["circuit_flux_linkage_Wb"], fsol.flux[i], rtol=1e-6,
                                   atol=1e-6 * np.abs(fsol.flux[i]).max())
        np.testing.assert_allclose(r["airgap_radial_flux_density_T"], fres.radial_b[i], rtol=0,
                                   atol=1e-6 * np.abs(fres.radial_b[i]).max())
        assert r["airgap_sample_angles_deg"] == angles
        # tangent block: library tangent on the periodic operator, reconstruction rules
        ssol = splan.solve([currents[i]])
        da, db1, db2, dflux, info = tplan.solve_tangent(ssol.a[0], currents[i], [[1.0, 0.0, 0.0]])
        t = spp.tangent(ssol.b1[0], ssol.b2[0], da, db1, db2)
        rhs = r["tangent_multi_rhs"]["rhs"][0]
        assert r["tangent_multi_rhs"]["status"] == "PASS"
        for got, want in ((rhs["dFx_N_per_A"], 2 * t.force[0, 0]), (rhs["dFy_N_per_A"], 2 * t.force[0, 1])):
            assert abs(got - want) <= 1e-6 * max(abs(want), 1e-9), (got, want)
        assert rhs["dtorque_Nm_per_A"] == 0.0
        part = np.array(dflux[0]) + (-1) * np.array(dflux[0])  # partner orientation -1, repeat sign +1
        np.testing.assert_allclose(rhs["circuit_flux_linkage_derivative_Wb_per_A"], part, atol=1e-12)
        np.testing.assert_allclose(rhs["airgap_radial_flux_density_derivative_T_per_A"], t.radial_b[0], rtol=0,
                                   atol=1e-6 * np.abs(t.radial_b[0]).max())


def test_batch_over_several_artifacts_shares_one_launch_and_equals_separate_batches(gpu, tmp_path):
    """Items on two posed artifacts in one chunk are solved in one multi-plan launch per
    Newton step (a replica plan for the second sample of an artifact); each item agrees with
    a batch of its artifact alone (per-artifact batched launch) to 1e-9."""
    path, _, source = motor_artifact(tmp_path)
    src = json.load(open(path))
    src["resolved"]["pose"] = {"rotor_angle_deg": 5, "displacement_mm": [0, 0]}
    other = tmp_path / "motor5.gpu.json"
    other.write_text(json.dumps(src))
    items = [{"task_id": "a0", "request": motor_request(path, source, [12.0])},
             {"task_id": "b0", "request": motor_request(other, source, [12.0], rotor_angle_deg=5)},
             {"task_id": "a1", "request": motor_request(path, source, [-4.0])}]
    rc, both, err = call(tmp_path, "--motor-batch", {"protocol": "gpu_femm_motor_batch_v1",
                                                     "max_items_per_chunk": 4, "items": items}, name="both.json")
    assert rc == 0 and both["status"] == "PASS", err
    for k, item in enumerate(items):
        rc, alone, err = call(tmp_path, "--motor-batch", {"protocol": "gpu_femm_motor_batch_v1",
                                                          "max_items_per_chunk": 4, "items": [item]},
                              name=f"alone{k}.json")
        assert rc == 0, err
        got, want = both["items"][k]["response"], alone["items"][0]["response"]
        for key in ("torque_Nm", "Fx_N", "Fy_N"):
            assert abs(got[key] - want[key]) <= 1e-9 * max(abs(want["torque_Nm"]), abs(want["Fx_N"]), 1e-12), key
        f, w = np.array(got["circuit_flux_linkage_Wb"]), np.array(want["circuit_flux_linkage_Wb"])
        assert np.linalg.norm(f - w) <= 1e-9 * np.linalg.norm(w)
