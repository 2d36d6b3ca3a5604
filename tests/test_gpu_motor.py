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
