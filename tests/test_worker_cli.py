"""femm_gpu --worker, the streaming batch worker (MotorBatchWorker, gpu_solver/src/app/
motor_worker.cpp:24-191), on the CPU: the job envelope and its refusals with the
reference's error strings, session / sequence rules (a refused job still consumes its
number), one status line per job, responses published for the jobs that run.  Without a
GPU the jobs that run end with GPU_UNAVAILABLE items; the solved responses are checked in
test_gpu_worker.py."""
import hashlib
import json
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN, ROOT

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
SESSION = hashlib.sha256(b"session-a").hexdigest()


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def sample(art, cur):
    return {"protocol": "gpu_femm_magnetostatic_sample_v1", "mesh_artifact_path": str(art),
            "mesh_artifact_sha256": sha(art), "circuit_currents_A": [cur], "force_group_number": -1,
            "stress_air_group_number": -1, "airgap_radius_mm": 0, "airgap_angles_deg": [],
            "sliding_band_angle_deg": 0, "compute_force_torque": False, "include_field_solution": False}


def batch_file(tmp_path, name, art, currents):
    b = {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 8,
         "items": [{"task_id": f"t{i}", "request": sample(art, c)} for i, c in enumerate(currents)]}
    p = tmp_path / name
    p.write_text(json.dumps(b))
    return p


def envelope(seq, request, response, session=SESSION, digest=None):
    return json.dumps({"session": session, "sequence": seq, "request_path": str(request),
                       "response_path": str(response), "request_sha256": digest or sha(request)})


def run_worker(lines, timeout=600):
    r = subprocess.run([CLI, "--worker"], input="\n".join(lines) + "\n", capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stderr
    return [json.loads(x) for x in r.stdout.strip().splitlines()]


@pytest.fixture
def art(tmp_path):
    a = tmp_path / "strip.gpu.json"
    shutil.copy(os.path.join(GOLDEN, "periodic_strip.gpu.json"), a)
    return a


def test_envelope_refusals_and_sequence(tmp_path, art):
    b1 = batch_file(tmp_path, "b1.json", art, [12.0, -3.0])
    big = batch_file(tmp_path, "big.json", art, [1.0] * 33)
    out = tmp_path / "out"
    out.mkdir()
    lines = [
        "{not json",                                                     # 1: consumes nothing
        json.dumps({"session": SESSION, "sequence": 1}),                 # envelope keys
        envelope(1, b1, out / "r1.json", session=SESSION.upper()),       # identity: upper-case hex
        envelope(0, b1, out / "r0.json"),                                # identity: sequence < 1
        envelope(1, b1, b1),                                             # unsafe: overwrites request
        envelope(1, b1, out / "r1.json", digest="0" * 64),               # request SHA mismatch
        envelope(2, big, out / "big.json"),                              # > 32 items
        envelope(3, b1, art),                                            # overwrites the artifact
        envelope(4, b1, out / "r4.json"),                                # runs
        envelope(6, b1, out / "r6.json"),                                # out of sequence
        envelope(5, b1, out / "r5.json", session=hashlib.sha256(b"b").hexdigest()),  # other session
        envelope(5, b1, out / "r5.json"),                                # runs
    ]
    st = run_worker(lines)
    assert len(st) == len(lines)
    errors = [s["error"] for s in st]
    assert errors[0] == errors[1] == "invalid stream job envelope"
    assert errors[2] == errors[3] == "invalid stream job identity"
    assert errors[4] == "unsafe stream output path"
    assert errors[5] == "stream request SHA-256 mismatch"
    assert errors[6] == "stream transaction exceeds 32 items"
    assert errors[7] == "stream response would overwrite an artifact"
    assert errors[8] == "" and errors[11] == ""
    assert errors[9] == errors[10] == "stream session or submission sequence mismatch"
    assert all(s["exit_code"] == 1 for s in st[:8]) and st[9]["exit_code"] == 1
    assert [s["sequence"] for s in st[8:]] == [4, 6, 5, 5]
    # The jobs that ran published a batch response; no other response files exist.
    assert sorted(os.listdir(out)) == ["r4.json", "r5.json"]
    body = json.load(open(out / "r4.json"))
    assert body["protocol"] == "gpu_femm_magnetostatic_batch_v1" and len(body["items"]) == 2
    assert [i["task_id"] for i in body["items"]] == ["t0", "t1"]
    for s in st:
        assert s["prepare_begin_seconds"] <= s["prepare_end_seconds"] <= s["solve_end_seconds"] + 1e-9
        assert s["session"] in (SESSION, SESSION.upper(), hashlib.sha256(b"b").hexdigest(), "")
