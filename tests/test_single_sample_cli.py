"""femm_gpu --single-sample on the CPU: the gpu_femm_single_sample_v1 request reader
against the reference's own ReadSingleSampleRequest (oracle/_ref, sample_request.cpp:
98-135) on well-formed and malformed requests, and the response envelope of the refusals
(WriteSingleSampleResponse, reference_adapter.cu:16-61).  The solved response is checked
on the GPU (test_gpu_postprocess.py)."""
import json
import os
import subprocess

import pytest

import oracle as O
from conftest import GOLDEN, ROOT

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
STEM = os.path.join(GOLDEN, "nonlinear_pm_coil_planar")
SHA = "f95e0c8f73850e3534117eac9a0988fdbcb37a73fe80b41fe0d8e3e18cb7d09c"
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")


def base(**kw):
    fields = [("protocol", '"gpu_femm_single_sample_v1"'), ("stem", json.dumps(STEM)),
              ("curve_directory", json.dumps(GOLDEN)), ("source_motor_fem_sha256", json.dumps(SHA)),
              ("current_A", "5"), ("selected_material_label", "1"), ("airgap_radius_mm", "1"),
              ("airgap_angles_deg", "[0, 90, 180, 270]")]
    fields = [(k, kw.get(k, v)) for k, v in fields]
    return "{\n" + ",\n".join(f'  "{k}": {v}' for k, v in fields if v is not None) + "\n}\n"


VARIANTS = {
    "golden": base(),
    "wrong protocol": base(protocol='"gpu_femm_single_sample_v2"'),
    "label 2": base(selected_material_label="2"),
    "label 1.5": base(selected_material_label="1.5"),
    "label hex float": base(selected_material_label="0x1p0"),
    "short sha": base(source_motor_fem_sha256=json.dumps(SHA[:-1])),
    "non-hex sha": base(source_motor_fem_sha256=json.dumps("g" + SHA[1:])),
    "upper-case sha": base(source_motor_fem_sha256=json.dumps(SHA.upper())),
    "angles without radius": base(airgap_radius_mm="0"),
    "negative radius": base(airgap_radius_mm="-1", airgap_angles_deg="[]"),
    "no angles": base(airgap_angles_deg="[]"),
    "trailing comma": base(airgap_angles_deg="[0, 90,]"),
    "missing comma": base(airgap_angles_deg="[0 90]"),
    "nan angle": base(airgap_angles_deg="[nan]"),
    "string current": base(current_A='"5"'),
    "exponent current": base(current_A="5e0"),
    "infinite current": base(current_A="1e999"),
    "backslash stem": base(stem=json.dumps(STEM + "\\x")),
    "missing key": base(curve_directory=None),
    "empty stem": base(stem='""'),
}


def run(tmp_path, text):
    rq, rs = tmp_path / "req.json", tmp_path / "resp.json"
    rq.write_text(text)
    r = subprocess.run([CLI, "--single-sample", str(rq), str(rs)], capture_output=True, text=True, timeout=600)
    return r.returncode, json.loads(rs.read_text()), r.stderr, rq


@needs_ref
@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_request_reader_matches_the_reference(tmp_path, name):
    rc, body, err, rq = run(tmp_path, VARIANTS[name])
    ok, ref = O.ref_read_single_sample_request(rq)
    assert body["protocol"] == "gpu_femm_single_sample_v1"
    if not ok:
        assert rc == 1 and body["status"] == "FAIL"
        assert body["error_identifier"] == "GPU_FEMM_INVALID_ARGUMENT" and body["source_motor_fem_sha256"] == ""
        assert f"FAIL single-sample request: {ref}" in err
        assert body["Fx_N"] is None and body["convergence"] == {"iterations": 0, "residual_l2": None}
        return
    # Accepted by both: the response echoes the request's SHA; without a GPU it is a
    # GPU_UNAVAILABLE failure, with one a solved response.
    assert body["source_motor_fem_sha256"] == ref["source_motor_fem_sha256"]
    assert body["status"] == "PASS" or body["error_identifier"] == "GPU_FEMM_GPU_UNAVAILABLE", body
    if body["status"] == "PASS":
        assert body["airgap_sample_angles_deg"] == ref["airgap_angles_deg"]


def test_missing_fixture_is_an_input_error(tmp_path):
    rc, body, err, _ = run(tmp_path, base(stem=json.dumps(str(tmp_path / "absent"))))
    assert rc == 1 and body["error_identifier"] == "GPU_FEMM_INPUT_IO" and body["error_message"] == "INPUT_IO"
    assert body["source_motor_fem_sha256"] == SHA
    assert "FAIL single-sample reference: invalid nonlinear [Solution] node count" in err
