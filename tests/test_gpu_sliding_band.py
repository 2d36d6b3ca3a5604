"""GPU tests of the sliding-band motor protocols: a gpu_femm_mesh_v2 artifact solved at
several rotor angles through --motor-single-sample and --motor-batch (tangent blocks
included), against the reference's own CPU path on the same posed model (oracle/_ref:
ApplySlidingBandAngle, the reference host assembler with FEMM's PCG, and
ComputeAirGapElementPostprocess / ComputeAirGapElementTangentPostprocess).

Tolerances (both sides at the reference's production options, whose own
production-to-tight drift on these models is 4e-9 in flux and 8e-8 in A):
* flux linkage within 1e-7 relative (2-norm); torque within 1e-6 relative; force within
  1e-6 of the force scale |torque| / r_gap (the two-pole rotor's net force is round-off);
  air-gap radial B within 1e-6 of its largest sample;
* tangent derivatives: dflux within 1e-6 relative, dtorque within 1e-5 of the torque-per-amp
  scale |torque| / max|current|, radial dB within 1e-5 of its largest sample (each side
  linearises at its own converged field).
"""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from conftest import ROOT
from femm_gpu_b200 import meshes
from test_postprocess_host import model_from_description
from test_sliding_band_cli import BASE, SOURCE, describe_at, sliding_artifact_text

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built")
CLI = os.path.join(ROOT, "femm-gpu_b200", "bin", "femm_gpu")
R_GAP = 0.0455
PROBES = [0.0, 30.0, 95.0, 180.0, 271.5]


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def artifact(tmp_path_factory):
    d = tmp_path_factory.mktemp("v2")
    text = sliding_artifact_text(meshes.sliding_band_machine(nr=40, nt=30))
    path = d / "v2.json"
    path.write_text(text)
    return path, text, hashlib.sha256(text.encode()).hexdigest()


def request(path, sha, currents, angle, protocol="gpu_femm_motor_sample_v1", **kw):
    r = {"protocol": protocol, "mesh_artifact_path": str(path), "mesh_artifact_sha256": sha,
         "base_motor_fem_sha256": BASE, "source_fem_sha256": SOURCE,
         "circuit_currents_A": [float(c) for c in currents], "selected_group_number": 20, "air_group_number": 50,
         "airgap_radius_mm": 1e3 * R_GAP, "airgap_angles_deg": PROBES, "rotor_angle_deg": angle,
         "displacement_mm": [0, 0]}
    if protocol == "gpu_femm_motor_sample_v2":
        r["tangent_multi_rhs"] = None
    r.update(kw)
    return r


def call(tmp_path, command, body, name="in.json"):
    rq, rs = tmp_path / name, tmp_path / ("out_" + name)
    rq.write_text(json.dumps(body))
    r = subprocess.run([CLI, command, str(rq), str(rs)], capture_output=True, text=True, timeout=600)
    return r.returncode, json.loads(rs.read_text()), r.stderr


def reference(path, text, angle, currents):
    """The reference CPU path on the artifact posed at `angle`: (posed fg.Model, a, flux,
    (status, Fx, Fy, torque, radial))."""
    hp = O.ref_sliding_band_pose(O.ref_artifact_handle(text.encode()), angle)
    rc, d = describe_at(path, angle)
    assert rc == 0
    model = model_from_description(d)
    model.ages = [fg.AirGap(nodes=np.array(g["nodes"]).reshape(-1, 4), weights=np.array(g["weights"]).reshape(-1, 4),
                            inner_radius_m=g["ri_m"], outer_radius_m=g["ro_m"], arc_length_deg=g["arc_length_deg"],
                            inner_shift=g["inner_shift"], outer_shift=g["outer_shift"],
                            antiperiodic=bool(g["antiperiodic"]), center_m=tuple(g["center_m"]))
                  for g in d["air_gap_elements"]]
    a, flux, status, _ = O.ref_artifact_cpu_solve(hp, np.atleast_2d(currents), model.node_count,
                                                  model.circuit_count, threads=2)
    assert status[0] == 0
    post = O.ref_age_postprocess(hp, a[0], np.radians(PROBES))
    assert post[0] == 0
    return model, hp, a[0], flux[0], post


def check_base(resp, ref_flux, post):
    _, fx, fy, tq, radial = post
    assert resp["status"] == "PASS", resp
    assert rel(resp["circuit_flux_linkage_Wb"], ref_flux) <= 1e-7
    assert abs(resp["torque_Nm"] - tq) <= 1e-6 * abs(tq)
    scale = abs(tq) / R_GAP
    assert abs(resp["Fx_N"] - fx) <= 1e-6 * scale and abs(resp["Fy_N"] - fy) <= 1e-6 * scale
    radial = np.asarray(radial)
    assert np.max(np.abs(np.array(resp["airgap_radial_flux_density_T"]) - radial)) <= 1e-6 * np.abs(radial).max()
    assert resp["airgap_sample_angles_deg"] == PROBES


@needs_ref
@pytest.mark.parametrize("angle", [0.0, 12.5])
def test_single_sample_matches_reference_cpu_path(gpu, tmp_path, artifact, angle):
    path, text, sha = artifact
    cur = [8.0, -4.0, -4.0]
    rc, resp, err = call(tmp_path, "--motor-single-sample", request(path, sha, cur, angle))
    assert rc == 0, err
    _, _, _, flux, post = reference(path, text, angle, cur)
    check_base(resp, flux, post)


def ref_tangent(model, a, currents, directions):
    """dA of the consistent Jacobian at a (the reference's assembly, band included; the
    per-amp circuit loads from the restatement, which the band does not change), then the
    reference's band derivatives postprocess is applied by the caller."""
    plain = fg.Model(**{k: getattr(model, k) for k in model.__dataclass_fields__ if k != "ages"})
    sources = O.assemble(plain, a, currents, 1).sources
    system = O.assemble(model, a, currents, 1, use_ref=True)
    out = []
    for d in directions:
        rhs = sum(s * src for s, src in zip(d, sources))
        st, x, _, _ = O.pcg(system, rhs, tol=1e-13)
        assert st == 0
        da = np.where(system.node_to_free >= 0, system.node_sign * x[np.maximum(system.node_to_free, 0)], 0.0)
        _, _, dflux = O.finalize(plain, da)
        out.append((da, dflux))
    return out


@needs_ref
def test_batch_over_rotor_angles_with_tangents(gpu, tmp_path, artifact):
    path, text, sha = artifact
    dirs = {"d0": [1.0, 0.0, 0.0], "mix": [0.5, -0.25, 0.25]}
    tangent = {"schema_version": "gpu_femm_tangent_multi_rhs_v1",
               "rhs": [{"name": k, "circuit_current_derivative_A_per_A": v} for k, v in dirs.items()]}
    items = []
    plan = [(0.0, [8.0, -4.0, -4.0], False), (12.5, [8.0, -4.0, -4.0], True), (12.5, [-3.0, 6.0, -3.0], False),
            (33.0, [5.0, 1.0, -6.0], True)]
    for i, (angle, cur, with_tangent) in enumerate(plan):
        r = request(path, sha, cur, angle, protocol="gpu_femm_motor_sample_v2")
        if with_tangent:
            r["tangent_multi_rhs"] = tangent
        items.append({"task_id": f"t{i}", "request": r})
    body = {"protocol": "gpu_femm_motor_batch_v2", "max_items_per_chunk": 8, "items": items}
    rc, resp, err = call(tmp_path, "--motor-batch", body, name="batch.json")
    assert rc == 0 and resp["status"] == "PASS", err
    # one operator per rotor angle: three groups in the one chunk
    assert resp["cache"]["chunk_count"] == 1 and resp["cache"]["actual_parallel_width"] == 2
    for (angle, cur, with_tangent), item in zip(plan, resp["items"]):
        out = item["response"]
        model, hp, a, flux, post = reference(path, text, angle, cur)
        check_base(out, flux, post)
        if not with_tangent:
            assert "tangent_multi_rhs" not in out
            continue
        t = out["tangent_multi_rhs"]
        assert t["status"] == "PASS" and [r["name"] for r in t["rhs"]] == list(dirs)
        for (da, dflux), r in zip(ref_tangent(model, a, cur, dirs.values()), t["rhs"]):
            st, dfx, dfy, dtq, dradial = O.ref_age_tangent_postprocess(hp, a, da, np.radians(PROBES))
            assert st == 0
            assert rel(r["circuit_flux_linkage_derivative_Wb_per_A"], dflux) <= 1e-6
            assert abs(r["dtorque_Nm_per_A"] - dtq) <= 1e-5 * abs(post[3]) / np.max(np.abs(cur))
            dr = np.asarray(dradial)
            assert np.max(np.abs(np.array(r["airgap_radial_flux_density_derivative_T_per_A"]) - dr)) <= \
                1e-5 * np.abs(dr).max()


@needs_ref
def test_library_band_postprocess_on_device_solutions(gpu, artifact):
    """fg_air_gap_postprocess on the library's own solve of a posed model equals the reference
    postprocess of that same solution (the same field, so only rounding apart)."""
    path, text, _ = artifact
    model, hp, _, _, _ = reference(path, text, 7.0, [8.0, -4.0, -4.0])
    plan = fg.Plan(model)
    sol = plan.solve(meshes.seeded_currents(3, 3, 10.0, seed=8))
    got = plan.air_gap_postprocess(sol.a, np.radians(PROBES))
    for k in range(3):
        st, fx, fy, tq, radial = O.ref_age_postprocess(hp, sol.a[k], np.radians(PROBES))
        assert st == 0 and got.status[k] == 0
        assert abs(got.torque[k] - tq) <= 1e-12 * abs(tq)
        scale = abs(tq) / R_GAP
        assert abs(got.force[k, 0] - fx) <= 1e-12 * scale and abs(got.force[k, 1] - fy) <= 1e-12 * scale
        assert np.max(np.abs(got.radial_b[k] - radial)) <= 1e-12 * np.abs(radial).max()


@needs_ref
def test_native_sector_batch_matches_the_reference_path(gpu, tmp_path):
    """gpu_femm_motor_batch_v4 on the 180-degree anti-periodic native air-gap element sector of
    the two-pole machine, against the reference CPU path on the same posed sector with the
    reference's reconstruction rules (torque x k, flux through the cyclic partner map,
    probes folded into [0, span) with the anti-periodic sign; batch_response.cpp:38-99,
    sample_request.cpp:568-599), to the base tolerances above.

    The reference's ApplySlidingBandAngle copies point 0's inner records into the band's
    closing point, which on an anti-periodic sector drops the -1 copy sign that record
    carries in FEMM's own records: the reference's torque and probes on such a sector are
    not the full machine's, and the library reproduces the reference.  At rotor angle 0
    the stiffness does not read that record (the inner corners sit on ring nodes), so the
    flux linkages there equal the full sliding-band machine's (1e-6)."""
    from test_sliding_band_cli import native_sector_artifact_text
    sec = meshes.sliding_band_machine(nr=40, nt=30, sector=True)
    stext = native_sector_artifact_text(sec)
    spath = tmp_path / "v4.json"
    spath.write_text(stext)
    ssha = hashlib.sha256(stext.encode()).hexdigest()
    cases = [(0.0, [8.0, -4.0, -4.0]), (12.5, [8.0, -4.0, -4.0]), (33.0, [5.0, 1.0, -6.0])]
    items = []
    for i, (angle, cur) in enumerate(cases):
        r = request(spath, ssha, cur, angle, protocol="gpu_femm_motor_sample_v4")
        r["tangent_multi_rhs"] = None
        r["sector_performance"] = {"schema_version": "gpu_femm_motor_sector_performance_v2",
                                   "model_invariance_certificate_sha256": "d" * 64}
        items.append({"task_id": f"s{i}", "request": r})
    rc, sresp, err = call(tmp_path, "--motor-batch", {"protocol": "gpu_femm_motor_batch_v4",
                                                      "max_items_per_chunk": 8, "items": items}, name="s.json")
    assert rc == 0 and sresp["status"] == "PASS", err
    for (angle, cur), item in zip(cases, sresp["items"]):
        s = item["response"]
        block = s["sector_reconstruction"]
        assert block["schema_version"] == "gpu_femm_motor_sector_reconstruction_v2"
        assert block["load_extraction_method"] == "native_air_gap_element_signed_sector"
        assert block["operator_construction"] == "native_age_sector_base_only"
        assert block["base_torque_multiplier"] == 2 and block["status"] == "PASS"
        assert s["Fx_N"] == 0.0 and s["Fy_N"] == 0.0
        hp = O.ref_sliding_band_pose(O.ref_artifact_handle(stext.encode()), angle)
        a, flux, st, _ = O.ref_artifact_cpu_solve(hp, [cur], sec.node_count, 3, threads=2)
        assert st[0] == 0
        folded, signs = [], []
        for deg in PROBES:
            t = np.radians(deg)
            copy = int(np.floor(t / np.pi))
            folded.append(t - copy * np.pi)
            signs.append(-1.0 if copy % 2 else 1.0)
        pst, _, _, tq, radial = O.ref_age_postprocess(hp, a[0], folded)
        assert pst == 0
        assert abs(s["torque_Nm"] - 2.0 * tq) <= 1e-6 * abs(2.0 * tq)
        full_flux = flux[0] + (-1.0) * (-1.0) * flux[0]  # partner c, orientation -1, anti-periodic
        assert rel(s["circuit_flux_linkage_Wb"], full_flux) <= 1e-7
        ref_radial = np.array(signs) * radial
        assert np.max(np.abs(np.array(s["airgap_radial_flux_density_T"]) - ref_radial)) <= \
            1e-6 * np.abs(ref_radial).max()
        if angle == 0.0:
            full = meshes.sliding_band_machine(nr=40, nt=30)
            _, full_flux_machine, st, _ = O.ref_artifact_cpu_solve(O.ref_model_handle(full), [cur],
                                                                   full.node_count, 3)
            assert st[0] == 0 and rel(s["circuit_flux_linkage_Wb"], full_flux_machine[0]) <= 1e-6


def planar_request(path, sha, currents, band_deg, **kw):
    r = {"protocol": "gpu_femm_planar_dc_sample_v1", "mesh_artifact_path": str(path), "mesh_artifact_sha256": sha,
         "circuit_currents_A": [float(c) for c in currents], "force_group_number": 20,
         "stress_air_group_number": 50, "airgap_radius_mm": 1e3 * R_GAP, "airgap_angles_deg": PROBES,
         "sliding_band_angle_deg": band_deg, "compute_force_torque": True, "include_field_solution": False}
    r.update(kw)
    return r


@needs_ref
def test_planar_dc_solve_and_batch_on_a_sliding_band_artifact(gpu, tmp_path, artifact):
    """The planar-DC adapter serves sliding-band artifacts as the reference does
    (sample_adapter.cpp:396-439): sliding_band_angle_deg poses the bands, the band
    postprocess answers; --solve equals --motor-single-sample at the same rotor angle bit for
    bit, and a batch over two band angles (solved side by side) equals its single solves to
    1e-7 (both converge to the production Newton tolerance)."""
    path, text, sha = artifact
    cur = [8.0, -4.0, -4.0]
    rc, s, err = call(tmp_path, "--solve", planar_request(path, sha, cur, 12.5), name="p.json")
    assert rc == 0 and s["status"] == "PASS", err
    rc, m, err = call(tmp_path, "--motor-single-sample", request(path, sha, cur, 12.5), name="m.json")
    assert rc == 0, err
    for key in ("Fx_N", "Fy_N", "torque_Nm", "circuit_flux_linkage_Wb", "airgap_radial_flux_density_T"):
        assert s[key] == m[key], key
    items = [{"task_id": f"i{i}", "request": planar_request(path, sha, c, a)}
             for i, (c, a) in enumerate([(cur, 12.5), ([-3.0, 6.0, -3.0], 0.0), (cur, 0.0)])]
    rc, b, err = call(tmp_path, "--batch", {"protocol": "gpu_femm_magnetostatic_batch_v1",
                                            "max_items_per_chunk": 8, "items": items}, name="b.json")
    assert rc == 0 and b["status"] == "PASS", err
    # the batch solves its two poses side by side (one multi-plan launch), converging within
    # the production Newton tolerance of --solve's own launch: 1e-7
    first = b["items"][0]["response"]
    assert abs(first["torque_Nm"] - s["torque_Nm"]) <= 1e-7 * abs(s["torque_Nm"])
    assert rel(first["circuit_flux_linkage_Wb"], s["circuit_flux_linkage_Wb"]) <= 1e-7
    _, _, _, flux, post = reference(path, text, 0.0, cur)
    check_base(b["items"][2]["response"], flux, post)
    # the probe circle must lie in the band
    rc, bad, _ = call(tmp_path, "--solve", planar_request(path, sha, cur, 0.0, airgap_radius_mm=47.0), name="x.json")
    assert rc == 1 and bad["status"] == "FAIL"


@needs_ref
def test_planar_dc_batch_joint_and_per_pose_paths_agree(gpu, tmp_path, artifact):
    """One planar-DC batch over two band angles, run down both paths: poses solved side by
    side in one multi-plan launch (max_items_per_chunk 8) and pose by pose
    (max_items_per_chunk 1).  Both meet the production Newton tolerance, so an item's
    answer depends on the path only below it: torque and flux linkage agree within 1e-7,
    and the 0-degree item matches the reference CPU path on both."""
    path, text, sha = artifact
    cases = [([8.0, -4.0, -4.0], 12.5), ([-3.0, 6.0, -3.0], 0.0), ([8.0, -4.0, -4.0], 0.0)]
    items = [{"task_id": f"i{i}", "request": planar_request(path, sha, c, a)} for i, (c, a) in enumerate(cases)]
    runs = []
    for chunk in (8, 1):
        rc, b, err = call(tmp_path, "--batch", {"protocol": "gpu_femm_magnetostatic_batch_v1",
                                                "max_items_per_chunk": chunk, "items": items},
                          name=f"chunk{chunk}.json")
        assert rc == 0 and b["status"] == "PASS", err
        runs.append([i["response"] for i in b["items"]])
    for joint, single in zip(*runs):
        assert abs(joint["torque_Nm"] - single["torque_Nm"]) <= 1e-7 * abs(single["torque_Nm"])
        assert rel(joint["circuit_flux_linkage_Wb"], single["circuit_flux_linkage_Wb"]) <= 1e-7
    _, _, _, flux, post = reference(path, text, 0.0, cases[2][0])
    for r in runs:
        check_base(r[2], flux, post)


@needs_ref
def test_sliding_band_transactions_in_the_worker(gpu, tmp_path, artifact):
    """Two worker transactions on one sliding-band artifact at different rotor angles (the
    artifact and its poses resident between jobs) answer as one-shot --motor-batch runs."""
    from test_worker_cli import envelope, run_worker
    path, _, sha = artifact
    bodies = []
    for j, angles in enumerate(((0.0, 12.5), (12.5, 40.0))):
        bodies.append({"protocol": "gpu_femm_motor_batch_v1", "max_items_per_chunk": 4,
                       "items": [{"task_id": f"j{j}i{i}", "request": request(path, sha, [8.0, -4.0, -4.0 + i], a)}
                                 for i, a in enumerate(angles)]})
    out = tmp_path / "out"
    out.mkdir()
    envs = []
    for j, body in enumerate(bodies):
        b = tmp_path / f"b{j}.json"
        b.write_text(json.dumps(body))
        envs.append(envelope(j + 1, b, out / f"w{j}.json"))
    st = run_worker(envs)
    assert all(s["exit_code"] == 0 and s["error"] == "" for s in st), st
    for j, body in enumerate(bodies):
        got = json.load(open(out / f"w{j}.json"))
        rc, ref, _ = call(tmp_path, "--motor-batch-profile", body, name=f"p{j}.json")
        assert rc == 0
        assert [i["response"] for i in got["items"]] == [i["response"] for i in ref["items"]]


@needs_ref
def test_worker_bounds_resident_poses_and_recreates_evicted_ones(gpu, tmp_path):
    """A worker meeting more rotor angles than it keeps resident (kResidentPoses = 64) trims
    the least recently used poses between chunks and rebuilds an evicted pose on demand:
    jobs over 70 angles, then a job revisiting evicted and resident angles, answer as
    one-shot runs."""
    from test_worker_cli import envelope, run_worker
    text = sliding_artifact_text(meshes.sliding_band_machine(nr=40, nt=12))
    path = tmp_path / "small_v2.json"
    path.write_text(text)
    sha = hashlib.sha256(text.encode()).hexdigest()
    angles = [0.5 * i for i in range(70)]
    # worker transactions carry at most 32 items: three jobs meet 70 angles, the fourth
    # (after the trim to 64 evicted the six oldest) revisits evicted and resident ones
    jobs = [angles[:32], angles[32:64], angles[64:], [0.0, 0.5, 1.5, 34.5]]
    bodies = [{"protocol": "gpu_femm_motor_batch_v1", "max_items_per_chunk": 32,
               "items": [{"task_id": f"j{j}i{i}", "request": request(path, sha, [8.0, -4.0, -4.0], a)}
                         for i, a in enumerate(js)]} for j, js in enumerate(jobs)]
    out = tmp_path / "out"
    out.mkdir()
    envs = []
    for j, body in enumerate(bodies):
        b = tmp_path / f"pose{j}.json"
        b.write_text(json.dumps(body))
        envs.append(envelope(j + 1, b, out / f"pose{j}.json"))
    st = run_worker(envs)
    assert all(s["exit_code"] == 0 for s in st), st
    for j, body in enumerate(bodies):
        got = json.load(open(out / f"pose{j}.json"))
        rc, ref, _ = call(tmp_path, "--motor-batch", body, name=f"one{j}.json")
        assert rc == 0 and got["status"] == "PASS"
        assert [i["response"] for i in got["items"]] == [i["response"] for i in ref["items"]]
