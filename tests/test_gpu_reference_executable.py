"""The reference's own GPU executable (gpu_linear_p1_poc built for sm_100a by oracle/Makefile's
refgpu target) as a second oracle of the JSON boundary: the same request files answered by
both executables.

* --solve on the stock-FEMM fixtures (periodic / anti-periodic strips, axisymmetric coil):
  same status, same Newton iteration count, flux linkage within 1e-10 relative, nodal
  potential within 1e-9 relative 2-norm (both are the FP64 Jacobi PCG method; the kernels
  differ in reduction order);
* --solve on a 14,641-node nonlinear planar square (iron B-H, magnet, 3 circuits): the same,
  with flux linkage within 1e-8 and potential within 1e-8 (production Newton gates);
* --motor-batch of four samples on a posed motor artifact: every item's status, flux
  linkage (1e-9), force and torque (1e-9 of the largest) agree.
"""
import hashlib
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from femm_gpu_b200 import artifact, meshes
from test_gpu_motor import BASE, motor_artifact, motor_request

pytestmark = pytest.mark.gpu

OURS = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
THEIRS = os.path.join(ROOT, "oracle", "_ref", "bin", "femm_gpu_ref")
needs_exe = pytest.mark.skipif(not os.path.exists(THEIRS), reason="reference GPU executable not built")


def request(path, currents, include=True):
    return {"protocol": "gpu_femm_magnetostatic_sample_v1", "mesh_artifact_path": str(path),
            "mesh_artifact_sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(),
            "circuit_currents_A": [float(c) for c in currents], "force_group_number": -1,
            "stress_air_group_number": -1, "airgap_radius_mm": 0, "airgap_angles_deg": [],
            "sliding_band_angle_deg": 0, "compute_force_torque": False, "include_field_solution": include}


def run(exe, tmp_path, command, body, name):
    rq, rs = tmp_path / f"{name}.in.json", tmp_path / f"{name}.{os.path.basename(exe)}.json"
    rq.write_text(json.dumps(body))
    r = subprocess.run([exe, command, str(rq), str(rs)], capture_output=True, text=True, timeout=900)
    return r.returncode, json.loads(rs.read_text()), r.stderr


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def compare_solve(tmp_path, path, currents, name, tol_flux, tol_a):
    rc1, ours, e1 = run(OURS, tmp_path, "--solve", request(path, currents), name)
    rc2, theirs, e2 = run(THEIRS, tmp_path, "--solve", request(path, currents), name)
    assert rc1 == rc2 == 0, (e1, e2)
    assert ours["status"] == theirs["status"] == "PASS"
    assert ours["solve_status"] == theirs["solve_status"]
    assert ours["convergence"]["iterations"] == theirs["convergence"]["iterations"]
    assert rel(ours["circuit_flux_linkage_Wb"], theirs["circuit_flux_linkage_Wb"]) <= tol_flux
    assert rel(ours["node_potential"], theirs["node_potential"]) <= tol_a
    return ours, theirs


@needs_exe
@pytest.mark.parametrize("name", ["periodic_strip", "antiperiodic_strip", "axisymmetric_coil"])
def test_stock_fixtures_answer_as_the_reference_executable(gpu, tmp_path, name):
    path = tmp_path / (name + ".gpu.json")
    shutil.copy(os.path.join(GOLDEN, name + ".gpu.json"), path)
    cur = json.load(open(os.path.join(GOLDEN, "expected.json")))[name]["circuit_current_A"]
    compare_solve(tmp_path, path, [cur], name, 1e-10, 1e-9)


@needs_exe
def test_nonlinear_square_answers_as_the_reference_executable(gpu, tmp_path):
    model = meshes.square_nonlinear(m=120, seed=2)
    text, _ = artifact.write_artifact(model, [0.0, 0.0, 0.0])
    path = tmp_path / "square120.gpu.json"
    path.write_text(text)
    for i, cur in enumerate(meshes.seeded_currents(2, 3, 20.0, seed=31)):
        compare_solve(tmp_path, path, cur, f"square{i}", 1e-8, 1e-8)


@needs_exe
def test_motor_batch_answers_as_the_reference_executable(gpu, tmp_path):
    path, _, source = motor_artifact(tmp_path)
    body = {"protocol": "gpu_femm_motor_batch_v1", "max_items_per_chunk": 4,
            "items": [{"task_id": f"t{i}", "request": motor_request(path, source, [c])}
                      for i, c in enumerate((12.0, -6.0, 3.0, 0.5))]}
    rc1, ours, e1 = run(OURS, tmp_path, "--motor-batch", body, "motor")
    rc2, theirs, e2 = run(THEIRS, tmp_path, "--motor-batch", body, "motor")
    assert rc1 == rc2 == 0, (e1, e2)
    assert ours["status"] == theirs["status"] == "PASS"
    assert [i["task_id"] for i in ours["items"]] == [i["task_id"] for i in theirs["items"]]
    for a, b in zip(ours["items"], theirs["items"]):
        a, b = a["response"], b["response"]
        assert a["status"] == b["status"] == "PASS"
        assert rel(a["circuit_flux_linkage_Wb"], b["circuit_flux_linkage_Wb"]) <= 1e-9
        scale = max(abs(b["Fx_N"]), abs(b["Fy_N"]), 1e-300)
        assert abs(a["Fx_N"] - b["Fx_N"]) <= 1e-9 * scale and abs(a["Fy_N"] - b["Fy_N"]) <= 1e-9 * scale
        assert abs(a["torque_Nm"] - b["torque_Nm"]) <= 1e-9 * max(abs(b["torque_Nm"]), 1e-300)
        assert a["base_motor_fem_sha256"] == b["base_motor_fem_sha256"] == BASE
