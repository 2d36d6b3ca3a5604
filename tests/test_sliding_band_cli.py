"""The sliding-band motor artifacts (gpu_femm_mesh_v2: a zero-degree reference mesh whose air
gap is native air-gap elements; gpu_femm_mesh_v4: one cyclic sector of it) on the CPU: parsing against the reference's own parser
(ParseGpuFemmMeshArtifactJson, oracle/_ref), the band records posed at rotor angles
against the reference's ApplySlidingBandAngle bit for bit, the parse refusals' messages,
and the motor requests the adapters refuse before any GPU work (RequestMatchesArtifact,
sample_request.cpp:393-446).  Solved sliding-band responses are checked in
test_gpu_sliding_band.py."""
import copy
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT
from femm_gpu_b200 import meshes
from test_cli_boundary import describe, ref_parse

CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
BASE = "b" * 64
SOURCE = "a" * 64


def sliding_artifact_text(model, base=BASE, source=SOURCE, as_object=False):
    """A gpu_femm_mesh_v2 artifact of a zero-degree sliding-band model
    (meshes.sliding_band_machine), its band written as the artifact's air_gap_elements."""
    from femm_gpu_b200 import artifact
    text, _ = artifact.write_artifact(model, [0.0] * model.circuit_count, source_sha256=source)
    root = json.loads(text)
    root["schema_version"] = "gpu_femm_mesh_v2"
    root["base_motor_fem_sha256"] = base
    res = root["resolved"]
    res["base_motor_fem_sha256"] = base
    res["pose"] = {"rotor_angle_deg": 0, "displacement_mm": [0, 0]}
    del res["node_constraints"]
    bands = []
    for i, g in enumerate(model.ages):
        pts = [{"n0": int(n[0]), "w0": float(w[0]), "n1": int(n[1]), "w1": float(w[1]), "n2": int(n[2]),
                "w2": float(w[2]), "n3": int(n[3]), "w3": float(w[3])} for n, w in zip(g.nodes, g.weights)]
        bands.append({"name": f"gap{i}", "periodicity": "antiperiodic" if g.antiperiodic else "periodic",
                      "center_mm": [1e3 * g.center_m[0], 1e3 * g.center_m[1]], "ri_mm": 1e3 * g.inner_radius_m,
                      "ro_mm": 1e3 * g.outer_radius_m, "arc_length_deg": g.arc_length_deg,
                      "sector_count": int(g.nodes.shape[0] - 1), "inner_shift": g.inner_shift,
                      "outer_shift": g.outer_shift, "quad_points": pts})
    res["air_gap_elements"] = bands[0] if as_object and len(bands) == 1 else bands
    return json.dumps(root)


def describe_at(path, angle):
    r = subprocess.run([CLI, "--describe-artifact", str(path), repr(float(angle))], capture_output=True, text=True,
                       timeout=120)
    return r.returncode, json.loads(r.stdout) if r.stdout.strip() else None


def assert_bands_equal(mine, theirs):
    assert len(mine) == len(theirs)
    for d, (meta, nodes, weights) in zip(mine, theirs):
        assert d["antiperiodic"] == int(meta[0])
        assert d["center_m"] == [meta[1], meta[2]] and d["ri_m"] == meta[3] and d["ro_m"] == meta[4]
        assert d["arc_length_deg"] == meta[5]
        assert d["inner_shift"] == meta[6] and d["outer_shift"] == meta[7]
        assert np.array_equal(np.array(d["nodes"]), nodes.ravel())
        assert np.array_equal(np.array(d["weights"]), weights.ravel())


@pytest.fixture(scope="module")
def band_model():
    return meshes.sliding_band_machine(nr=40, nt=30)


@needs_ref
@pytest.mark.parametrize("as_object", [False, True])
def test_sliding_artifact_parses_like_the_reference(tmp_path, band_model, as_object):
    text = sliding_artifact_text(band_model, as_object=as_object)
    p = tmp_path / "v2.json"
    p.write_text(text)
    rc, d = describe(str(p))
    ref, err = ref_parse(text.encode())
    assert rc == 0 and ref is not None, (d, err)
    assert np.array_equal(np.array(d["xy"]), ref["xy"]) and np.array_equal(np.array(d["tri"]), ref["tri"])
    assert np.array_equal(np.array(d["tri_mat"]), ref["tm"])
    mats = np.array(d["materials"])
    assert np.array_equal(mats[:, :5], ref["md"].reshape(-1, 5))
    assert np.array_equal(mats[:, 5:].astype(int), ref["mi"].reshape(-1, 3))
    assert np.array_equal(np.array(d["dirichlet_nodes"]), ref["dn"])
    h = O.ref_artifact_handle(text.encode())
    assert_bands_equal(d["air_gap_elements"], O.ref_age_records(h))
    assert d["plan_status"] == "OK"


@needs_ref
def test_bands_posed_at_rotor_angles_equal_the_reference(tmp_path, band_model):
    text = sliding_artifact_text(band_model)
    p = tmp_path / "v2.json"
    p.write_text(text)
    h = O.ref_artifact_handle(text.encode())
    # within one arc, across arcs, negative, beyond a turn, exactly on a ring node
    for angle in (0.0, 2.5, 6.0, 7.3, 40.0, -13.7, 725.25, 359.999):
        rc, d = describe_at(p, angle)
        assert rc == 0, d
        assert_bands_equal(d["air_gap_elements"], O.ref_age_records(O.ref_sliding_band_pose(h, angle)))
        assert d["plan_status"] == "OK"
    rc, d = describe_at(p, float("nan"))
    assert rc == 1 and d["status"] == "FAIL"


@needs_ref
def test_posed_reference_mesh_matches_a_turned_mesh(tmp_path, band_model):
    """Sliding the zero-degree bands by an angle gives the records of a mesh whose rotor is
    turned by that angle (the same ring nodes in the same order)."""
    text = sliding_artifact_text(band_model)
    h = O.ref_artifact_handle(text.encode())
    turned = meshes.sliding_band_machine(nr=40, nt=30, rotor_deg=7.3)
    meta, nodes, weights = O.ref_age_records(O.ref_sliding_band_pose(h, 7.3))[0]
    assert np.array_equal(nodes, turned.ages[0].nodes)
    assert abs(meta[6] - turned.ages[0].inner_shift) < 1e-12


@needs_ref
def test_sliding_artifact_refusals_follow_the_reference(tmp_path, band_model):
    root = json.loads(sliding_artifact_text(band_model))
    gap = root["resolved"]["air_gap_elements"][0]

    def with_gap(**kw):
        v = copy.deepcopy(root)
        v["resolved"]["air_gap_elements"][0].update(kw)
        return v

    variants = {"turned pose": copy.deepcopy(root), "moved pose": copy.deepcopy(root),
                "no band": copy.deepcopy(root), "band not a list": copy.deepcopy(root),
                "periodicity": with_gap(periodicity="none"), "one arc": with_gap(sector_count=1),
                "point count": with_gap(sector_count=gap["sector_count"] + 1),
                "center": with_gap(center_mm=[0]), "empty name": with_gap(name=""),
                "non-integer node": with_gap(quad_points=[dict(gap["quad_points"][0], n0=1.5)] + gap["quad_points"][1:]),
                "point member": with_gap(quad_points=[{"n0": 0}] + gap["quad_points"][1:]),
                "node out of range": with_gap(quad_points=[dict(gap["quad_points"][0], n2=10 ** 7)]
                                              + gap["quad_points"][1:]),
                "extra band member": with_gap(extra=1)}
    variants["turned pose"]["resolved"]["pose"]["rotor_angle_deg"] = 5
    variants["moved pose"]["resolved"]["pose"]["displacement_mm"] = [0, 0.1]
    variants["no band"]["resolved"]["air_gap_elements"] = []
    variants["band not a list"]["resolved"]["air_gap_elements"] = 3
    p = tmp_path / "bad.json"
    for label, v in variants.items():
        text = json.dumps(v)
        p.write_text(text)
        rc, d = describe(str(p))
        ref, ref_err = ref_parse(text.encode())
        assert ref is None and rc == 1, label
        assert d["error"] == ref_err, (label, d["error"], ref_err)
    # a v2 body under the native sector schema lacks its sector fields, as the reference says
    v = copy.deepcopy(root)
    v["schema_version"] = "gpu_femm_mesh_v4"
    text = json.dumps(v)
    p.write_text(text)
    rc, d = describe(str(p))
    ref, ref_err = ref_parse(text.encode())
    assert rc == 1 and ref is None and d["error"] == ref_err


def sample_request(artifact_path, sha, **kw):
    req = {"protocol": "gpu_femm_motor_sample_v1", "mesh_artifact_path": str(artifact_path),
           "mesh_artifact_sha256": sha, "base_motor_fem_sha256": BASE, "source_fem_sha256": SOURCE,
           "circuit_currents_A": [8.0, -4.0, -4.0], "selected_group_number": 20, "air_group_number": 50,
           "airgap_radius_mm": 45.5, "airgap_angles_deg": [0.0, 45.0, 90.0], "rotor_angle_deg": 12.5,
           "displacement_mm": [0, 0]}
    req.update(kw)
    return req


@needs_ref
def test_sliding_requests_refused_before_any_gpu_work(tmp_path, band_model):
    import hashlib
    text = sliding_artifact_text(band_model)
    art = tmp_path / "v2.json"
    art.write_text(text)
    sha = hashlib.sha256(text.encode()).hexdigest()
    cases = {"displaced": dict(displacement_mm=[0.1, 0]), "absent selected group": dict(selected_group_number=7),
             "absent air group": dict(air_group_number=8), "circle inside the rotor": dict(airgap_radius_mm=44.0),
             "circle beyond the stator side": dict(airgap_radius_mm=46.5),
             "circuit count": dict(circuit_currents_A=[1.0, 2.0]), "source identity": dict(source_fem_sha256="c" * 64)}
    for label, kw in cases.items():
        rq, rs = tmp_path / "rq.json", tmp_path / "rs.json"
        rq.write_text(json.dumps(sample_request(art, sha, **kw)))
        r = subprocess.run([CLI, "--motor-single-sample", str(rq), str(rs)], capture_output=True, text=True,
                           timeout=120)
        body = json.loads(rs.read_text())
        assert r.returncode == 1 and body["status"] == "FAIL", label
        assert body["solve_status"] == "INVALID_ARGUMENT", (label, body["solve_status"])


def native_sector_artifact_text(model, cert="d" * 64, **sector):
    """A gpu_femm_mesh_v4 artifact of a native air-gap element sector
    (meshes.sliding_band_machine(sector=True)): the v2 writing plus the sector metadata and
    the anti-periodic edge constraints."""
    root = json.loads(sliding_artifact_text(model))
    root["schema_version"] = "gpu_femm_mesh_v4"
    res = root["resolved"]
    res["node_constraints"] = [{"node_a": int(a), "node_b": int(b), "relation": "antiperiodic" if s < 0 else "periodic"}
                               for a, b, s in zip(model.con_a, model.con_b, model.con_sign)]
    meta = {"schema_version": "gpu_femm_motor_sector_v2", "sector_start_angle_deg": 0, "angle_deg": 180,
            "full_machine_sector_count": 2, "electrical_pole_pairs": 1, "suspension_spatial_order": 2,
            "boundary_relation": "antiperiodic", "circuit_partner_indices": list(range(model.circuit_count)),
            "circuit_partner_orientations": [-1] * model.circuit_count, "apex_self_pair_nodes": [],
            "model_invariance_certificate_sha256": cert}
    meta.update(sector)
    res["sector"] = meta
    return json.dumps(root)


@pytest.fixture(scope="module")
def sector_model():
    return meshes.sliding_band_machine(nr=40, nt=30, sector=True)


@needs_ref
def test_native_sector_artifact_parses_like_the_reference(tmp_path, sector_model):
    text = native_sector_artifact_text(sector_model)
    p = tmp_path / "v4.json"
    p.write_text(text)
    rc, d = describe(str(p))
    ref, err = ref_parse(text.encode())
    assert rc == 0 and ref is not None, (d, err)
    assert np.array_equal(np.array(d["xy"]), ref["xy"]) and np.array_equal(np.array(d["tri_mat"]), ref["tm"])
    assert np.array_equal(np.array(d["dirichlet_nodes"]), ref["dn"])
    nc = ref["sizes"][5]
    con = ref["con"][: 3 * nc].reshape(-1, 3)
    assert np.array_equal(np.array(d["constraint_nodes"]).reshape(-1, 2), con[:, :2])
    assert np.array_equal(np.array(d["constraint_signs"]), con[:, 2])
    h = O.ref_artifact_handle(text.encode())
    assert_bands_equal(d["air_gap_elements"], O.ref_age_records(h))
    for angle in (3.0, 45.5, -20.0):
        rc, d = describe_at(p, angle)
        assert rc == 0 and d["plan_status"] == "OK"
        assert_bands_equal(d["air_gap_elements"], O.ref_age_records(O.ref_sliding_band_pose(h, angle)))


@needs_ref
def test_native_sector_refusals_follow_the_reference(tmp_path, sector_model):
    variants = {
        "sector schema": dict(schema_version="gpu_femm_motor_sector_v1"),
        "angle": dict(angle_deg=120),
        "phase advance": dict(full_machine_sector_count=4, angle_deg=90),
        "relation parity": dict(boundary_relation="periodic"),
        "partner closure": dict(circuit_partner_indices=[1, 0, 2], circuit_partner_orientations=[1, -1, -1]),
    }
    p = tmp_path / "bad.json"
    texts = {k: native_sector_artifact_text(sector_model, **kw) for k, kw in variants.items()}
    root = json.loads(native_sector_artifact_text(sector_model))
    v = copy.deepcopy(root)
    v["resolved"]["air_gap_elements"] = []
    texts["no band"] = json.dumps(v)
    v = copy.deepcopy(root)
    v["resolved"]["air_gap_elements"][0]["periodicity"] = "periodic"
    texts["band periodicity"] = json.dumps(v)
    v = copy.deepcopy(root)
    v["resolved"]["air_gap_elements"][0]["arc_length_deg"] = 360
    texts["band arc"] = json.dumps(v)
    v = copy.deepcopy(root)
    v["resolved"]["node_constraints"][0]["node_b"] = v["resolved"]["node_constraints"][1]["node_b"]
    texts["pair not a sector rotation"] = json.dumps(v)
    for label, text in texts.items():
        p.write_text(text)
        rc, d = describe(str(p))
        ref, ref_err = ref_parse(text.encode())
        assert ref is None and rc == 1, label
        assert d["error"] == ref_err, (label, d["error"], ref_err)


@needs_ref
def test_planar_dc_requests_on_sliding_artifacts_refused_before_any_gpu_work(tmp_path, band_model):
    """PlanarDcRequestMatchesArtifact (sample_adapter.cpp:181-234) on a sliding-band
    artifact: the probe circle must lie in the band, and the generic protocol does not take
    motor artifacts."""
    import hashlib
    text = sliding_artifact_text(band_model)
    art = tmp_path / "v2.json"
    art.write_text(text)
    sha = hashlib.sha256(text.encode()).hexdigest()
    base = {"protocol": "gpu_femm_planar_dc_sample_v1", "mesh_artifact_path": str(art), "mesh_artifact_sha256": sha,
            "circuit_currents_A": [8.0, -4.0, -4.0], "force_group_number": 20, "stress_air_group_number": 50,
            "airgap_radius_mm": 45.5, "airgap_angles_deg": [0.0, 90.0], "sliding_band_angle_deg": 7.5,
            "compute_force_torque": True, "include_field_solution": False}
    cases = {"circle outside the band": dict(airgap_radius_mm=47.0),
             "absent force group": dict(force_group_number=9),
             "generic protocol": dict(protocol="gpu_femm_magnetostatic_sample_v1", force_group_number=-1,
                                      stress_air_group_number=-1, airgap_radius_mm=0, airgap_angles_deg=[],
                                      compute_force_torque=False, sliding_band_angle_deg=0)}
    for label, kw in cases.items():
        rq, rs = tmp_path / "rq.json", tmp_path / "rs.json"
        rq.write_text(json.dumps(dict(base, **kw)))
        r = subprocess.run([CLI, "--solve", str(rq), str(rs)], capture_output=True, text=True, timeout=120)
        body = json.loads(rs.read_text())
        assert r.returncode == 1 and body["status"] == "FAIL", label
        assert body["error_message"] == "artifact physics, circuit count, group, or sliding-band request mismatch", \
            (label, body["error_message"])
