"""GPU test of femm_gpu --worker: responses of streamed jobs equal the one-shot --batch
responses of the same batch files (the worker keeps plans and masks resident between jobs
but solves with the same code), and an artifact file changed under a resident plan fails
its items exactly as --batch does."""
import hashlib
import json
import os
import shutil
import subprocess

import pytest

from conftest import GOLDEN
from test_gpu_postprocess import legacy_artifact, sample as planar_sample
from test_worker_cli import CLI, batch_file, envelope, run_worker, sha

pytestmark = pytest.mark.gpu


def one_shot(tmp_path, request):
    out = tmp_path / ("oneshot_" + os.path.basename(request))
    r = subprocess.run([CLI, "--batch", str(request), str(out)], capture_output=True, text=True, timeout=600)
    return r.returncode, json.load(open(out))


def strip_fields(body):
    return [(i["task_id"], i["response"]["status"], i["response"]["circuit_flux_linkage_Wb"],
             i["response"].get("Fx_N"), i["response"]["error_message"]) for i in body["items"]]


def test_worker_matches_one_shot_batches(gpu, tmp_path):
    per = tmp_path / "per.gpu.json"
    anti = tmp_path / "anti.gpu.json"
    shutil.copy(os.path.join(GOLDEN, "periodic_strip.gpu.json"), per)
    shutil.copy(os.path.join(GOLDEN, "antiperiodic_strip.gpu.json"), anti)
    legacy, _ = legacy_artifact(tmp_path)
    b1 = batch_file(tmp_path, "b1.json", per, [12.0, -3.0, 7.5])
    b2 = batch_file(tmp_path, "b2.json", per, [1.0, 2.0])
    b3 = batch_file(tmp_path, "b3.json", anti, [12.0])
    post = {"protocol": "gpu_femm_magnetostatic_batch_v1", "max_items_per_chunk": 4,
            "items": [{"task_id": f"p{i}", "request": planar_sample(legacy, [c], compute_force_torque=True,
                                                                     force_group_number=2,
                                                                     stress_air_group_number=0)}
                      for i, c in enumerate((12.0, -6.0))]}
    b4 = tmp_path / "b4.json"
    b4.write_text(json.dumps(post))
    b5 = tmp_path / "b5.json"
    b5.write_text(json.dumps(post))
    out = tmp_path / "out"
    out.mkdir()
    files = [b1, b2, b3, b4, b5]
    st = run_worker([envelope(i + 1, f, out / f"r{i + 1}.json") for i, f in enumerate(files)])
    assert [s["exit_code"] for s in st] == [0] * 5 and all(s["error"] == "" for s in st)
    for i, f in enumerate(files):
        rc, ref = one_shot(tmp_path, f)
        got = json.load(open(out / f"r{i + 1}.json"))
        assert rc == 0 and got["status"] == ref["status"] == "PASS"
        assert strip_fields(got) == strip_fields(ref)


def test_changed_artifact_fails_like_one_shot(gpu, tmp_path):
    per = tmp_path / "per.gpu.json"
    shutil.copy(os.path.join(GOLDEN, "periodic_strip.gpu.json"), per)
    b1 = batch_file(tmp_path, "b1.json", per, [12.0])
    out = tmp_path / "out"
    out.mkdir()
    # The second job names the original SHA, but the file changed in between.
    proc = subprocess.Popen([CLI, "--worker"], stdin=subprocess.PIPE, stdout=subprocess.PIPE, text=True)
    proc.stdin.write(envelope(1, b1, out / "r1.json") + "\n")
    proc.stdin.flush()
    first = json.loads(proc.stdout.readline())
    per.write_text(per.read_text() + " ")
    proc.stdin.write(envelope(2, b1, out / "r2.json") + "\n")
    proc.stdin.close()
    second = json.loads(proc.stdout.readline())
    assert proc.wait(timeout=600) == 0
    assert first["exit_code"] == 0 and second["exit_code"] == 1 and second["error"] == ""
    body = json.load(open(out / "r2.json"))
    assert body["items"][0]["response"]["error_message"] == "mesh artifact SHA mismatch"
    rc, ref = one_shot(tmp_path, b1)
    assert rc == 1 and strip_fields(ref) == strip_fields(body)
