"""GPU tests of the femm_gpu CLI (--solve, --batch) on the reference's stock-FEMM fixtures.

Tolerances: flux linkage within the reference's own fixture gates (1e-10 relative for the
periodic / anti-periodic strips, 1e-3 for the axisymmetric coil, tests/native/
reference_commands.cu) and within 1e-12 of the library's fg_solve_batch on the same
artifact (the CLI adds no arithmetic); batch items within 1e-9 of the same sample solved
alone (a wider batch runs a different kernel shape); the mixed / block-Jacobi options
within the mixed-form bound 1e-8.
"""
import hashlib
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import femm_gpu_b200 as fg
from conftest import GOLDEN, ROOT
from femm_gpu_b200 import artifact

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
EXPECTED = json.load(open(os.path.join(GOLDEN, "expected.json")))
GATES = {"periodic_strip": 1e-10, "antiperiodic_strip": 1e-10, "axisymmetric_coil": 1e-3}


def request(path, currents, include=False, **kw):
    r = {"protocol": "gpu_femm_magnetostatic_sample_v1", "mesh_artifact_path": str(path),
         "mesh_artifact_sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(),
         "circuit_currents_A": list(map(float, currents)), "force_group_number": -1,
         "stress_air_group_number": -1, "airgap_radius_mm": 0, "airgap_angles_deg": [],
         "sliding_band_angle_deg": 0, "compute_force_torque": False, "include_field_solution": include}
    r.update(kw)
    return r


def call(tmp_path, command, body, *options):
    rq = tmp_path / "in.json"
    rq.write_text(json.dumps(body))
    rs = tmp_path / "out.json"
    r = subprocess.run([CLI, *options, command, str(rq), str(rs)], capture_output=True, text=True,
                       timeout=600)
    return r.returncode, json.loads(rs.read_text()), r.stderr


def copy_fixture(tmp_path, name):
    dst = tmp_path / (name + ".gpu.json")
    shutil.copy(os.path.join(GOLDEN, name + ".gpu.json"), dst)
    return dst


@pytest.mark.parametrize("name", sorted(GATES))
def test_solve_matches_stock_femm_and_the_library(gpu, tmp_path, name):
    path = copy_fixture(tmp_path, name)
    cur = EXPECTED[name]["circuit_current_A"]
    rc, body, err = call(tmp_path, "--solve", request(path, [cur], include=True))
    assert rc == 0, err
    assert body["status"] == "PASS" and body["solve_status"] == "OK"
    assert body["postprocess_status"] == "NOT_REQUESTED"
    flux = body["circuit_flux_linkage_Wb"][0]
    exp = EXPECTED[name]["flux_linkage_Wb"]
    assert abs(flux - exp) <= GATES[name] * abs(exp)
    model, _ = artifact.read_artifact(str(path))
    got = fg.Plan(model).solve([[cur]])
    assert abs(flux - got.flux[0, 0]) <= 1e-12 * abs(got.flux[0, 0])
    assert body["mesh_node_count"] == model.node_count and body["mesh_element_count"] == model.tri_count
    pot = np.array(body["node_potential"])
    if model.problem_type == fg.AXISYMMETRIC:
        assert body["problem_type"] == "axisymmetric" and body["field_components"] == ["Br", "Bz"]
        np.testing.assert_allclose(pot, got.a[0] * 2 * np.pi * model.xy[:, 0], rtol=1e-12, atol=1e-300)
    else:
        np.testing.assert_allclose(pot, got.a[0], rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(body["element_B_component_1_T"], got.b1[0], rtol=1e-12, atol=1e-15)
    assert body["convergence"]["iterations"] == got.info[0].iterations


def test_batch_groups_artifacts_and_keeps_order(gpu, tmp_path):
    per = copy_fixture(tmp_path, "periodic_strip")
    anti = copy_fixture(tmp_path, "antiperiodic_strip")
    items = [("p0", per, 12.0), ("a0", anti, 12.0), ("p1", per, -3.0), ("p2", per, 7.5),
             ("a1", anti, 1.0), ("p3", per, 0.25)]
    batch = {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 3,
             "items": [{"task_id": t, "request": request(p, [c])} for t, p, c in items]}
    rc, body, err = call(tmp_path, "--batch", batch)
    assert rc == 0, err
    assert body["status"] == "PASS" and body["cache"]["mesh_cache_hits"] == 4
    assert body["cache"]["chunk_count"] == 3  # periodic: 3 + 1, anti-periodic: 2
    assert [i["task_id"] for i in body["items"]] == [t for t, _, _ in items]
    for (t, p, c), item in zip(items, body["items"]):
        rc1, single, _ = call(tmp_path, "--solve", request(p, [c]))
        assert rc1 == 0 and item["response"]["status"] == "PASS"
        f, g = item["response"]["circuit_flux_linkage_Wb"][0], single["circuit_flux_linkage_Wb"][0]
        assert abs(f - g) <= 1e-9 * abs(g), t


def test_solver_options_mixed_block_jacobi(gpu, tmp_path):
    path = copy_fixture(tmp_path, "periodic_strip")
    rc, plain, _ = call(tmp_path, "--solve", request(path, [12.0]))
    rc2, fast, err = call(tmp_path, "--solve", request(path, [12.0]), "--preconditioner", "block-jacobi",
                          "--precision", "mixed")
    assert rc == rc2 == 0, err
    f, g = fast["circuit_flux_linkage_Wb"][0], plain["circuit_flux_linkage_Wb"][0]
    assert abs(f - g) <= 1e-8 * abs(g)


def test_generic_protocol_refuses_postprocess_requests(gpu, tmp_path):
    # The generic protocol exposes only the field solve (sample_adapter.cpp:199-205).
    path = copy_fixture(tmp_path, "periodic_strip")
    rc, body, _ = call(tmp_path, "--solve", request(path, [12.0], compute_force_torque=True))
    assert rc == 1 and body["status"] == "FAIL" and body["solve_status"] == "INVALID_ARGUMENT"
    assert body["postprocess_status"] == "NOT_RUN" and body["Fx_N"] is None
