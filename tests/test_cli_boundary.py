"""The JSON request / response boundary (femm-gpu_b200/bin/femm_gpu) on the CPU.

* The C++ artifact parser maps the reference fixtures onto exactly the model the
  reference's own parser builds (oracle/_ref, ParseGpuFemmMeshArtifactJson), bit for bit,
  and rejects the same malformed artifacts.
* SHA-256 of file bytes agrees with hashlib on the padding boundaries.
* --solve / --batch error paths follow the reference adapter (sample_adapter.cpp:407-489):
  request validation, artifact SHA binding, circuit-count match, no overwriting of the
  request or the artifact, atomic publication (no temporary file left behind).  Without a
  GPU a valid request ends in GPU_UNAVAILABLE; the solved responses are checked by the GPU
  tests (tests/test_gpu_cli.py).
"""
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

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
FIXTURES = ["periodic_strip", "antiperiodic_strip", "axisymmetric_coil"]


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120)


def describe(path):
    r = run("--describe-artifact", path)
    return r.returncode, json.loads(r.stdout) if r.stdout.strip() else None


def ref_parse(text: bytes):
    R = O.ref()
    h = C.c_void_p()
    rc = R.ref_parse_artifact(text, C.c_size_t(len(text)), C.byref(h))
    if rc != 0:
        err = R.ref_artifact_error(h).decode() if h else ""
        if h:
            R.ref_artifact_free(h)
        return None, err
    sizes = np.zeros(8, np.int32)
    depth, ptype = C.c_double(), C.c_int32()
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    R.ref_artifact_sizes(h, p(sizes), C.byref(depth), C.byref(ptype))
    N, E, M = sizes[:3]
    out = dict(xy=np.zeros(2 * N), tri=np.zeros(3 * E, np.int32), tm=np.zeros(E, np.int32),
               md=np.zeros(5 * M), mi=np.zeros(3 * M, np.int32), cb=np.zeros(max(sizes[7], 1)),
               dn=np.zeros(sizes[4], np.int32), con=np.zeros(3 * max(sizes[5], 1), np.int32),
               cu=np.zeros(max(sizes[6], 1)))
    ch, cs = np.zeros_like(out["cb"]), np.zeros_like(out["cb"])
    R.ref_artifact_copy(h, p(out["xy"]), p(out["tri"]), p(out["tm"]), p(out["md"]), p(out["mi"]),
                        p(out["cb"]), p(ch), p(cs), p(out["dn"]), p(out["con"]), p(out["cu"]))
    R.ref_artifact_free(h)
    out["ch"] = ch
    out["sizes"] = sizes
    out["depth"], out["ptype"] = depth.value, ptype.value
    return out, ""


needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("name", FIXTURES)
def test_parser_builds_the_reference_model(name):
    path = os.path.join(GOLDEN, name + ".gpu.json")
    text = open(path, "rb").read()
    rc, d = describe(path)
    assert rc == 0 and d["status"] == "PASS" and d["plan_status"] == "OK"
    ref, err = ref_parse(text)
    assert ref is not None, err
    assert d["sha256"] == hashlib.sha256(text).hexdigest()
    assert np.array_equal(np.array(d["xy"]), ref["xy"])
    assert np.array_equal(np.array(d["tri"]), ref["tri"]) and np.array_equal(np.array(d["tri_mat"]), ref["tm"])
    mats = np.array(d["materials"])
    md, mi = ref["md"].reshape(-1, 5), ref["mi"].reshape(-1, 3)
    assert np.array_equal(mats[:, :5], md)  # nu0, alpha, J per amp, Hc, angle: bit for bit
    assert np.array_equal(mats[:, 5:].astype(int), mi)  # curve, circuit, group
    npts = ref["sizes"][7]
    if npts:
        b = np.concatenate([c[0] for c in d["curves"]])
        h = np.concatenate([c[1] for c in d["curves"]])
        assert np.array_equal(b, ref["cb"][:npts]) and np.array_equal(h, ref["ch"][:npts])
    assert np.array_equal(np.array(d["dirichlet_nodes"]), ref["dn"])
    nc = ref["sizes"][5]
    con = ref["con"][: 3 * nc].reshape(-1, 3)
    assert np.array_equal(np.array(d["constraint_nodes"]).reshape(-1, 2), con[:, :2].reshape(-1, 2))
    assert np.array_equal(np.array(d["constraint_signs"]), con[:, 2])
    assert d["depth_m"] == ref["depth"] and d["problem_type"] == ref["ptype"]
    assert np.array_equal(np.array(d["circuit_currents_A"]), ref["cu"][: ref["sizes"][6]])


def tampered(text: str):
    """Malformed variants of an artifact: (label, text)."""
    root = json.loads(text)
    out = [("trailing data", text + " x"),
           ("duplicate key", text.replace('"schema_version"', '"schema_version": "x", "schema_version"', 1)),
           ("unicode escape", text.replace('"name": "', '"name": "\\u0041', 1)),
           ("leading zero", text.replace('"frequency_hz": 0', '"frequency_hz": 00', 1)),
           ("truncated", text[: len(text) // 2])]
    bad = json.loads(text)
    bad["resolved"]["model"]["depth_mm"] = 2 * float(bad["resolved"]["model"]["depth_mm"])
    out.append(("identity mismatch", json.dumps(bad)))
    bad = json.loads(text)
    bad["schema_version"] = "gpu_femm_mesh_v9"
    out.append(("unknown schema", json.dumps(bad)))
    bad = json.loads(text)
    del bad["resolved"]["circuits"]
    out.append(("missing field", json.dumps(bad)))
    assert root  # the original parses
    return out


@needs_ref
@pytest.mark.parametrize("name", FIXTURES)
def test_malformed_artifacts_are_rejected_like_the_reference(name, tmp_path):
    text = open(os.path.join(GOLDEN, name + ".gpu.json")).read()
    for label, bad in tampered(text):
        p = tmp_path / "bad.json"
        p.write_text(bad)
        rc, d = describe(str(p))
        ref, ref_err = ref_parse(bad.encode())
        assert ref is None, label
        assert rc == 1 and d["status"] == "FAIL", label
        if label not in ("unknown schema",):
            assert d["error"] == ref_err, (label, d["error"], ref_err)


@pytest.mark.parametrize("n", [0, 3, 55, 56, 63, 64, 65, 119, 200])
def test_sha256_padding_boundaries(n, tmp_path):
    data = bytes((7 * i + 3) % 256 for i in range(n))
    p = tmp_path / "f.bin"
    p.write_bytes(data)
    r = run("--sha256", str(p))
    assert r.returncode == 0 and r.stdout.strip() == hashlib.sha256(data).hexdigest()


def request(artifact_path, currents, protocol="gpu_femm_magnetostatic_sample_v1", include=False, **kw):
    sha = hashlib.sha256(open(artifact_path, "rb").read()).hexdigest()
    r = {"protocol": protocol, "mesh_artifact_path": str(artifact_path), "mesh_artifact_sha256": sha,
         "circuit_currents_A": list(currents), "force_group_number": -1, "stress_air_group_number": -1,
         "airgap_radius_mm": 0, "airgap_angles_deg": [], "sliding_band_angle_deg": 0,
         "compute_force_torque": False, "include_field_solution": include}
    r.update(kw)
    return r


@pytest.fixture
def strip(tmp_path):
    art = tmp_path / "strip.gpu.json"
    shutil.copy(os.path.join(GOLDEN, "periodic_strip.gpu.json"), art)
    return art


def solve(tmp_path, req, name="resp.json"):
    rq = tmp_path / "req.json"
    rq.write_text(json.dumps(req) if not isinstance(req, str) else req)
    rs = tmp_path / name
    r = run("--solve", str(rq), str(rs))
    body = json.loads(rs.read_text()) if rs.exists() else None
    leftovers = [f for f in os.listdir(tmp_path) if ".tmp." in f]
    assert not leftovers
    return r.returncode, body


def test_solve_request_errors(strip, tmp_path):
    rc, body = solve(tmp_path, "{not json")
    assert rc == 1 and body["status"] == "FAIL" and body["solve_status"] == "INVALID_ARGUMENT"
    assert body["protocol"] == "gpu_femm_planar_dc_sample_v1"
    req = request(strip, [12.0])
    req["extra"] = 1
    rc, body = solve(tmp_path, req)
    assert rc == 1 and body["solve_status"] == "INVALID_ARGUMENT"
    rc, body = solve(tmp_path, request(strip, [12.0], mesh_artifact_sha256="0" * 64))
    assert rc == 1 and body["error_message"] == "mesh artifact SHA mismatch"
    rc, body = solve(tmp_path, request(strip, [12.0, 1.0]))
    assert rc == 1 and body["solve_status"] == "INVALID_ARGUMENT"
    assert "circuit count" in body["error_message"]
    # the legacy planar-DC protocol does not accept a generic artifact
    rc, body = solve(tmp_path, request(strip, [12.0], protocol="gpu_femm_planar_dc_sample_v1"))
    assert rc == 1 and body["solve_status"] == "INVALID_ARGUMENT"
    rc, body = solve(tmp_path, request(tmp_path / "missing.json", [12.0], mesh_artifact_sha256="a" * 64)
                     if False else request(strip, [12.0], mesh_artifact_path=str(tmp_path / "missing.json")))
    assert rc == 1 and body["solve_status"] == "INPUT_IO"


def test_solve_never_overwrites_request_or_artifact(strip, tmp_path):
    rq = tmp_path / "req.json"
    rq.write_text(json.dumps(request(strip, [12.0])))
    before = rq.read_text()
    r = run("--solve", str(rq), str(rq))
    assert r.returncode == 1 and rq.read_text() == before
    art_before = strip.read_bytes()
    r = run("--solve", str(rq), str(strip))
    assert r.returncode == 1 and strip.read_bytes() == art_before


def test_cli_usage_and_options():
    assert run().returncode == 2
    assert run("--preconditioner", "ilu", "--capabilities").returncode == 2
    caps = json.loads(run("--preconditioner", "block-jacobi", "--capabilities").stdout)
    assert "gpu_femm_magnetostatic_batch_v1" in caps["protocols"]


def test_batch_envelope_validation(strip, tmp_path):
    item = {"task_id": "a", "request": request(strip, [12.0])}
    for bad in ({"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 0, "items": [item]},
                {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 4, "items": [item, item]},
                {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 4,
                 "items": [{"task_id": "bad id", "request": item["request"]}]},
                {"protocol": "gpu_femm_motor_batch_v1", "max_items_per_chunk": 4, "items": [item]}):
        rq = tmp_path / "batch.json"
        rq.write_text(json.dumps(bad))
        rs = tmp_path / "out.json"
        r = run("--batch", str(rq), str(rs))
        body = json.loads(rs.read_text())
        assert r.returncode == 1 and body["status"] == "FAIL" and body["items"] == []
