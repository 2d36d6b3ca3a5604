"""The production motor protocols on the CPU: the posed motor artifact (gpu_femm_mesh_v1)
against the reference's own parser, gpu_femm_motor_sample_v1..v4 requests against the
reference's ReadMotorSampleRequestJson (oracle/_ref), the motor batch envelope rules
(batch_prepare.cpp:73-129), and the adapters' refusals (sample_adapter.cpp:135-179,
motor_batch.cpp:32-53).  Solved motor responses are checked in test_gpu_motor.py."""
import copy
import ctypes as C
import hashlib
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, ROOT
from test_cli_boundary import describe, ref_parse

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
MOTOR = os.path.join(GOLDEN, "motor_mesh_v1.gpu.json")
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
BASE = "b" * 64
SOURCE = "a" * 64


@needs_ref
def test_motor_artifact_parses_like_the_reference():
    text = open(MOTOR, "rb").read()
    rc, d = describe(MOTOR)
    ref, err = ref_parse(text)
    assert rc == 0 and ref is not None, err
    assert np.array_equal(np.array(d["xy"]), ref["xy"]) and np.array_equal(np.array(d["tri"]), ref["tri"])
    assert np.array_equal(np.array(d["tri_mat"]), ref["tm"])
    mats = np.array(d["materials"])
    assert np.array_equal(mats[:, :5], ref["md"].reshape(-1, 5))
    assert np.array_equal(mats[:, 5:].astype(int), ref["mi"].reshape(-1, 3))
    assert np.array_equal(np.array(d["dirichlet_nodes"]), ref["dn"])


@needs_ref
def test_motor_artifact_refusals_follow_the_reference(tmp_path):
    root = json.load(open(MOTOR))
    variants = []
    bad = copy.deepcopy(root)
    bad["resolved"]["pose"]["displacement_mm"] = [0.1]
    variants.append(("pose", bad))
    bad = copy.deepcopy(root)
    bad["resolved"]["base_motor_fem_sha256"] = "c" * 64
    variants.append(("base identity", bad))
    bad = copy.deepcopy(root)
    bad["resolved"]["model"]["problem_type"] = "axisymmetric"
    variants.append(("physics", bad))
    bad = copy.deepcopy(root)
    del bad["resolved"]["pose"]
    variants.append(("missing pose", bad))
    bad = copy.deepcopy(root)
    bad["resolved"]["node_constraints"] = []
    variants.append(("extra field", bad))
    for label, v in variants:
        text = json.dumps(v)
        p = tmp_path / "m.json"
        p.write_text(text)
        rc, d = describe(str(p))
        ref, ref_err = ref_parse(text.encode())
        assert ref is None and rc == 1, label
        assert d["error"] == ref_err, (label, d["error"], ref_err)
    # Upper-case digests are accepted by the motor schema (no canonical identity check).
    ok = copy.deepcopy(root)
    ok["base_motor_fem_sha256"] = ok["resolved"]["base_motor_fem_sha256"] = "B" * 64
    p = tmp_path / "upper.json"
    p.write_text(json.dumps(ok))
    assert describe(str(p))[0] == 0 and ref_parse(json.dumps(ok).encode())[0] is not None
    # Under the sliding-band (v2), conforming sector (v3) and native sector (v4) schemas the
    # v1 body lacks their fields, as the reference says.
    for schema in ("gpu_femm_mesh_v2", "gpu_femm_mesh_v3", "gpu_femm_mesh_v4"):
        v = copy.deepcopy(root)
        v["schema_version"] = schema
        p.write_text(json.dumps(v))
        rc, d = describe(str(p))
        ref, ref_err = ref_parse(json.dumps(v).encode())
        assert rc == 1 and ref is None
        assert d["error"] == ref_err, (schema, d["error"], ref_err)


def sector_artifact_text(model, base=BASE, source=SOURCE, cert="d" * 64, **sector):
    """A gpu_femm_mesh_v3 artifact of a 180-degree sector model (two_pole_machine)."""
    from femm_gpu_b200 import artifact
    text, _ = artifact.write_artifact(model, [0.0] * model.circuit_count, source_sha256=source)
    root = json.loads(text)
    root["schema_version"] = "gpu_femm_mesh_v3"
    root["base_motor_fem_sha256"] = base
    res = root["resolved"]
    res["base_motor_fem_sha256"] = base
    res["pose"] = {"rotor_angle_deg": 0, "displacement_mm": [0, 0]}
    res["air_gap_elements"] = []
    meta = {"schema_version": "gpu_femm_motor_sector_v1", "sector_start_angle_deg": 0, "angle_deg": 180,
            "full_machine_sector_count": 2, "electrical_pole_pairs": 1, "suspension_spatial_order": 2,
            "boundary_relation": "antiperiodic", "circuit_partner_indices": list(range(model.circuit_count)),
            "circuit_partner_orientations": [-1] * model.circuit_count, "apex_self_pair_nodes": [],
            "model_invariance_certificate_sha256": cert}
    meta.update(sector)
    res["sector"] = meta
    return json.dumps(root)


@needs_ref
def test_sector_artifact_parses_like_the_reference(tmp_path):
    from femm_gpu_b200 import meshes
    model = meshes.two_pole_machine(nr=12, nt=24)
    good = sector_artifact_text(model)
    p = tmp_path / "s.json"
    p.write_text(good)
    rc, d = describe(str(p))
    ref, err = ref_parse(good.encode())
    assert rc == 0 and ref is not None, (d, err)
    assert np.array_equal(np.array(d["xy"]), ref["xy"]) and np.array_equal(np.array(d["tri_mat"]), ref["tm"])
    assert np.array_equal(np.array(d["dirichlet_nodes"]), ref["dn"])
    nc = ref["sizes"][5]
    con = ref["con"][: 3 * nc].reshape(-1, 3)
    assert np.array_equal(np.array(d["constraint_signs"]), con[:, 2])
    variants = {
        "angle": dict(angle_deg=90),
        "count": dict(full_machine_sector_count=3),
        "order": dict(suspension_spatial_order=3),
        "relation parity": dict(boundary_relation="periodic"),
        "partner": dict(circuit_partner_indices=[0, 0, 2]),
        "orientation": dict(circuit_partner_orientations=[2, -1, -1]),
        "apex off origin": dict(apex_self_pair_nodes=[5]),
        "certificate": dict(model_invariance_certificate_sha256="D" * 64),
        "schema": dict(schema_version="gpu_femm_motor_sector_v2"),
    }
    for label, kw in variants.items():
        text = sector_artifact_text(model, **kw)
        p.write_text(text)
        rc, d = describe(str(p))
        ref, ref_err = ref_parse(text.encode())
        assert ref is None and rc == 1, label
        assert d["error"] == ref_err, (label, d["error"], ref_err)
    # a constraint pair that is not a 180-degree rotation
    root = json.loads(good)
    root["resolved"]["nodes_mm"][int(model.con_b[3])][0] += 0.5
    text = json.dumps(root)
    p.write_text(text)
    rc, d = describe(str(p))
    ref, ref_err = ref_parse(text.encode())
    assert ref is None and rc == 1 and d["error"] == ref_err


def motor_request(protocol="gpu_femm_motor_sample_v1", **kw):
    r = {"protocol": protocol, "mesh_artifact_path": MOTOR,
         "mesh_artifact_sha256": hashlib.sha256(open(MOTOR, "rb").read()).hexdigest(),
         "base_motor_fem_sha256": BASE, "source_fem_sha256": SOURCE, "circuit_currents_A": [2, -2],
         "selected_group_number": 20, "air_group_number": 50, "airgap_radius_mm": 0, "airgap_angles_deg": [],
         "rotor_angle_deg": 3, "displacement_mm": [0.1, 0]}
    if protocol != "gpu_femm_motor_sample_v1":
        r["tangent_multi_rhs"] = None
    if protocol in ("gpu_femm_motor_sample_v3", "gpu_femm_motor_sample_v4"):
        r["sector_performance"] = {"schema_version": "gpu_femm_motor_sector_performance_v1"
                                   if protocol.endswith("v3") else "gpu_femm_motor_sector_performance_v2",
                                   "model_invariance_certificate_sha256": "d" * 64}
    r.update(kw)
    return r


TANGENT = {"schema_version": "gpu_femm_tangent_multi_rhs_v1",
           "rhs": [{"name": "suspension_d", "circuit_current_derivative_A_per_A": [1, 0]},
                   {"name": "suspension_q", "circuit_current_derivative_A_per_A": [0, 1]}]}

REQUESTS = {
    "v1": motor_request(),
    "v2 no tangent": motor_request("gpu_femm_motor_sample_v2"),
    "v2 empty list": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs=[]),
    "v2 tangent": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs=TANGENT),
    "v2 missing tangent": {k: v for k, v in motor_request("gpu_femm_motor_sample_v2").items()
                           if k != "tangent_multi_rhs"},
    "v1 with tangent": motor_request(tangent_multi_rhs=TANGENT),
    "v3": motor_request("gpu_femm_motor_sample_v3"),
    "v4 tangent": motor_request("gpu_femm_motor_sample_v4", tangent_multi_rhs=TANGENT),
    "v9": motor_request("gpu_femm_motor_sample_v9"),
    "equal groups": motor_request(air_group_number=20),
    "negative group": motor_request(selected_group_number=-1),
    "fractional group": motor_request(selected_group_number=20.5),
    "short sha": motor_request(base_motor_fem_sha256="b" * 63),
    "upper sha": motor_request(base_motor_fem_sha256="B" * 64),
    "angles without radius": motor_request(airgap_angles_deg=[0, 90]),
    "no currents": motor_request(circuit_currents_A=[]),
    "string current": motor_request(circuit_currents_A=["2", -2]),
    "bad displacement": motor_request(displacement_mm=[0.1]),
    "empty path": motor_request(mesh_artifact_path=""),
    "tangent bad name": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs={
        "schema_version": "gpu_femm_tangent_multi_rhs_v1",
        "rhs": [{"name": "bad name", "circuit_current_derivative_A_per_A": [1, 0]}]}),
    "tangent duplicate": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs={
        "schema_version": "gpu_femm_tangent_multi_rhs_v1", "rhs": [TANGENT["rhs"][0], TANGENT["rhs"][0]]}),
    "tangent wrong length": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs={
        "schema_version": "gpu_femm_tangent_multi_rhs_v1",
        "rhs": [{"name": "d", "circuit_current_derivative_A_per_A": [1]}]}),
    "tangent too many": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs={
        "schema_version": "gpu_femm_tangent_multi_rhs_v1",
        "rhs": [{"name": f"d{i}", "circuit_current_derivative_A_per_A": [1, 0]} for i in range(9)]}),
    "tangent schema": motor_request("gpu_femm_motor_sample_v2", tangent_multi_rhs={
        "schema_version": "gpu_femm_tangent_multi_rhs_v2", "rhs": TANGENT["rhs"]}),
}


def ref_read(text):
    err = C.create_string_buffer(4096)
    rc = O.ref().ref_read_motor_sample_request(text.encode(), C.c_size_t(len(text.encode())), err)
    return rc == 0, err.value.decode()


def run(*args, **kw):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=300, **kw)


@needs_ref
@pytest.mark.parametrize("name", sorted(REQUESTS))
def test_motor_request_reader_matches_the_reference(tmp_path, name):
    text = json.dumps(REQUESTS[name])
    ok, ref_err = ref_read(text)
    rq, rs = tmp_path / "req.json", tmp_path / "resp.json"
    rq.write_text(text)
    r = run("--motor-single-sample", str(rq), str(rs))
    body = json.loads(rs.read_text())
    if not ok:
        assert r.returncode == 1 and body["solve_status"] == "INVALID_ARGUMENT"
        assert body["protocol"] == "gpu_femm_motor_sample_v1" and body["mesh_artifact_sha256"] == ""
        assert f"FAIL motor single-sample request: {ref_err}" in r.stderr
        return
    # Accepted: v1 / v2 match the fixture's pose and identities; without a GPU the solve
    # reports GPU_UNAVAILABLE, sector requests fail the artifact match.
    assert body["protocol"] == REQUESTS[name]["protocol"]
    if name in ("v3",):
        assert body["solve_status"] == "INVALID_ARGUMENT"
        assert "artifact identity, pose, or circuit-count mismatch" in r.stderr
    elif name == "upper sha":
        assert body["solve_status"] == "INVALID_ARGUMENT"  # the artifact's base digest is lower-case
    else:
        assert body["status"] == "PASS" or body["solve_status"] == "GPU_UNAVAILABLE", body


def test_motor_single_sample_gate(tmp_path):
    rq, rs = tmp_path / "req.json", tmp_path / "resp.json"
    for kw, status, message in [
        (dict(rotor_angle_deg=4), "INVALID_ARGUMENT", "artifact identity, pose, or circuit-count mismatch"),
        (dict(circuit_currents_A=[2]), "INVALID_ARGUMENT", "artifact identity, pose, or circuit-count mismatch"),
        (dict(mesh_artifact_sha256="0" * 64), "INVALID_ARGUMENT", "mesh artifact SHA mismatch"),
        (dict(mesh_artifact_path=str(tmp_path / "absent.json")), "INPUT_IO", "cannot open mesh artifact")]:
        rq.write_text(json.dumps(motor_request(**kw)))
        r = run("--motor-single-sample", str(rq), str(rs))
        body = json.loads(rs.read_text())
        assert r.returncode == 1 and body["solve_status"] == status and body["Fx_N"] is None
        assert f"FAIL motor single-sample: {message}" in r.stderr
        assert body["mesh_artifact_sha256"] == motor_request(**kw)["mesh_artifact_sha256"]
    # --single-sample hands a gpu_femm_motor_sample_v1 request to the motor adapter.
    rq.write_text(json.dumps(motor_request(rotor_angle_deg=4)))
    r = run("--single-sample", str(rq), str(rs))
    assert json.loads(rs.read_text())["protocol"] == "gpu_femm_motor_sample_v1" and r.returncode == 1


def batch(items, protocol="gpu_femm_motor_batch_v1", chunk=4):
    return {"protocol": protocol, "max_items_per_chunk": chunk,
            "items": [{"task_id": t, "request": r} for t, r in items]}


def test_motor_batch_envelope(tmp_path):
    rq, rs = tmp_path / "b.json", tmp_path / "out.json"
    v1 = motor_request()
    cases = [
        (batch([("a", v1), ("a", v1)]), "invalid or duplicate batch task_id"),
        (batch([("bad id", v1)]), "invalid or duplicate batch task_id"),
        (batch([("a", v1)], protocol="gpu_femm_motor_batch_v2"), "motor batch and item protocol versions must match"),
        (batch([("a", v1)], chunk=0), "invalid gpu_femm_motor_batch_v1 request"),
        (batch([]), "invalid gpu_femm_motor_batch_v1 request"),
        (batch([("a", motor_request(air_group_number=20))]), "invalid gpu_femm_motor_sample_v1 request"),
    ]
    for body, message in cases:
        rq.write_text(json.dumps(body))
        if rs.exists():
            rs.unlink()
        r = run("--motor-batch", str(rq), str(rs))
        assert r.returncode == 1 and f"FAIL motor batch request: {message}" in r.stderr, (message, r.stderr)
        assert not rs.exists()  # no trusted item identity: no response
    # A valid batch answers every item in order; the gate refuses mismatched items.
    rq.write_text(json.dumps(batch([("ok", v1), ("pose", motor_request(rotor_angle_deg=1)),
                                    ("sha", motor_request(mesh_artifact_sha256="0" * 64))], chunk=2)))
    r = run("--motor-batch-profile", str(rq), str(rs))
    body = json.loads(rs.read_text())
    assert r.returncode == 1 and [i["task_id"] for i in body["items"]] == ["ok", "pose", "sha"]
    assert body["items"][1]["response"]["solve_status"] == "INVALID_ARGUMENT"
    assert body["items"][2]["response"]["solve_status"] == "INVALID_ARGUMENT"
    assert body["items"][0]["response"]["solve_status"] in ("OK", "GPU_UNAVAILABLE")
    assert body["cache"]["chunk_count"] == 2 and body["cache"]["effective_chunk_size"] == 2
    assert body["timing"]["schema_version"] == "gpu_femm_motor_batch_timing_v1"
