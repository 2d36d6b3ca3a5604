"""gpu_femm_magnetostatic_mesh_v1 / gpu_femm_planar_dc_mesh_v1 artifacts in Python.

``read_artifact`` maps an artifact onto a ``Model`` the way the reference's
ParseGpuFemmMeshArtifactJson does (gpu_solver/src/io/mesh_artifact.cpp:14-715):
millimetres to metres, nu0 = 1 / (mu0 mu_x), one label material per region appended
after the base materials (group, circuit, PM angle, J = turns / region area), zero
outer Dirichlet nodes, signed periodic / anti-periodic node constraints.
``write_artifact`` produces such an artifact from a ``Model`` together with its
canonical identity hash (compact JSON, object keys in byte order, numbers as
written -- CanonicalJsonSha256, gpu_solver/src/io/strict_json.cpp:466-527).

The C++ library carries its own strict parser for the CLI boundary; this module is
the Python host-side mirror used to build requests and fixtures.
"""
from __future__ import annotations

import hashlib
import json
from typing import Tuple

import numpy as np

from .model import AXISYMMETRIC, MU0, PLANAR, Model


class Num(str):
    """A JSON number kept as its source text (canonical hashing needs the text)."""


def _loads(text: str):
    return json.loads(text, parse_float=Num, parse_int=Num)


def _canonical(value) -> str:
    if isinstance(value, Num):
        return str(value)
    if value is None:
        return "null"
    if value is True:
        return "true"
    if value is False:
        return "false"
    if isinstance(value, str):
        # Byte-wise escaping of the UTF-8 text; bytes >= 0x20 pass through unchanged
        # (carried as latin-1 code points so the final encode restores the bytes).
        escapes = {0x22: '\\"', 0x5C: "\\\\", 8: "\\b", 12: "\\f", 10: "\\n", 13: "\\r", 9: "\\t"}
        out = ['"']
        for ch in value.encode("utf-8"):
            if ch in escapes:
                out.append(escapes[ch])
            elif ch < 0x20:
                out.append("\\u00%02x" % ch)
            else:
                out.append(chr(ch))
        out.append('"')
        return "".join(out)
    if isinstance(value, list):
        return "[" + ",".join(_canonical(v) for v in value) + "]"
    if isinstance(value, dict):
        keys = sorted(value.keys(), key=lambda k: k.encode("utf-8"))
        return "{" + ",".join(_canonical(k) + ":" + _canonical(value[k]) for k in keys) + "}"
    raise TypeError(type(value))


def canonical_sha256(value) -> str:
    text = _canonical(value)
    return hashlib.sha256(text.encode("latin-1")).hexdigest()


def _f(x) -> float:
    return float(x)


def _i(x) -> int:
    v = float(x)
    if v != int(v):
        raise ValueError("expected an integer")
    return int(v)


def read_artifact(text_or_path: str) -> Tuple[Model, np.ndarray]:
    """Returns (model, circuit currents from the artifact)."""
    if not text_or_path.lstrip().startswith("{"):
        with open(text_or_path, "r", encoding="utf-8") as f:
            text_or_path = f.read()
    root = _loads(text_or_path)
    schema = root["schema_version"]
    if schema not in ("gpu_femm_magnetostatic_mesh_v1", "gpu_femm_planar_dc_mesh_v1"):
        raise ValueError(f"unsupported schema {schema}")
    res = root["resolved"]
    if canonical_sha256(res) != root["canonical_identity_sha256"]:
        raise ValueError("canonical artifact identity mismatch")
    model = res["model"]
    ptype = AXISYMMETRIC if model["problem_type"] == "axisymmetric" else PLANAR
    depth = _f(model["depth_mm"]) * 1e-3
    xy = np.array([[_f(p[0]) * 1e-3, _f(p[1]) * 1e-3] for p in res["nodes_mm"]])
    nu0, alpha, jpa, hc, deg, cidx, circ, grp, curves = [], [], [], [], [], [], [], [], []
    mat_lookup = {}
    for m in res["materials"]:
        mat_lookup[_i(m["id"])] = len(nu0)
        nu0.append(1.0 / (MU0 * _f(m["mu_x"])))
        alpha.append(0.0)
        jpa.append(0.0)
        hc.append(_f(m["H_c_A_per_m"]))
        deg.append(0.0)
        circ.append(-1)
        grp.append(-1)
        if m["B_T"]:
            cidx.append(len(curves))
            curves.append((np.array([_f(v) for v in m["B_T"]]), np.array([_f(v) for v in m["H_A_per_m"]])))
        else:
            cidx.append(-1)
    currents = np.array([_f(c["current_A"]) for c in res["circuits"]], dtype=np.float64)
    regions = []
    region_lookup = {}
    for r in res["regions"]:
        region_lookup[_i(r["id"])] = len(regions)
        regions.append((mat_lookup[_i(r["material_id"])], _i(r["circuit_index"]), _f(r["turns"]),
                        _f(r["pm_magnetization_deg"]), _i(r["group_number"])))
    faces = res["triangles"]["node_indices"]
    tri = np.array([[_i(v) for v in f] for f in faces], dtype=np.int64)
    treg = np.array([region_lookup[_i(v)] for v in res["triangles"]["region_ids"]], dtype=np.int64)
    area = np.zeros(len(regions))
    for e in range(tri.shape[0]):
        p0, p1, p2 = xy[tri[e, 0]], xy[tri[e, 1]], xy[tri[e, 2]]
        det = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1])
        if not det > 0.0:
            raise ValueError("triangle is not CCW")
        area[treg[e]] += 0.5 * det
    base = len(nu0)
    for k, (mat, circuit, turns, angle, group) in enumerate(regions):
        nu0.append(nu0[mat])
        alpha.append(alpha[mat])
        hc.append(hc[mat])
        cidx.append(cidx[mat])
        deg.append(angle)
        circ.append(circuit)
        grp.append(group)
        jpa.append(0.0 if circuit < 0 else turns / area[k])
    bnd = res["outer_dirichlet"]
    con = res.get("node_constraints", [])
    return Model(
        xy=xy, tri=tri.astype(np.int32), tri_mat=(base + treg).astype(np.int32),
        nu0=nu0, alpha=alpha, j_per_a=jpa, hc=hc, mag_deg=deg, curve_index=cidx,
        circuit_index=circ, group=grp, curves=curves,
        dir_nodes=[_i(v) for v in bnd["node_indices"]],
        dir_values=[_f(v) for v in bnd["A_Wb_per_m"]],
        con_a=[_i(c["node_a"]) for c in con], con_b=[_i(c["node_b"]) for c in con],
        con_sign=[1 if c["relation"] == "periodic" else -1 for c in con],
        circuit_count=len(currents), depth_m=depth, problem_type=ptype, name="artifact",
    ), currents


def _num(x: float) -> Num:
    return Num(repr(float(x)))


def write_artifact(model: Model, currents, source_sha256: str = "0" * 64) -> Tuple[str, str]:
    """Serialises a Model (one region per material label) as gpu_femm_magnetostatic_mesh_v1.

    Returns (json text, canonical identity sha256)."""
    mats, regions = [], []
    for i in range(model.mat_count):
        mu = 1.0 / (MU0 * model.nu0[i])
        b, h = (model.curves[model.curve_index[i]] if model.curve_index[i] >= 0 else ([], []))
        mats.append({"id": Num(str(i)), "name": f"m{i}", "mu_x": _num(mu), "mu_y": _num(mu),
                     "H_c_A_per_m": _num(model.hc[i]), "B_T": [_num(v) for v in b],
                     "H_A_per_m": [_num(v) for v in h], "lam_type": Num("0"), "lam_fill": Num("1")})
    tri_area = np.zeros(model.mat_count)
    p0, p1, p2 = model.xy[model.tri[:, 0]], model.xy[model.tri[:, 1]], model.xy[model.tri[:, 2]]
    det = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p2[:, 0] - p0[:, 0]) * (p1[:, 1] - p0[:, 1])
    np.add.at(tri_area, model.tri_mat, 0.5 * det)
    for i in range(model.mat_count):
        c = int(model.circuit_index[i])
        turns = model.j_per_a[i] * tri_area[i] if c >= 0 else 0.0
        regions.append({"id": Num(str(i)), "group_number": Num(str(max(int(model.group[i]), 0))),
                        "material_id": Num(str(i)), "circuit_index": Num(str(c)),
                        "turns": _num(turns), "pm_magnetization_deg": _num(model.mag_deg[i])})
    resolved = {
        "source_fem_sha256": source_sha256,
        "model": {"depth_mm": _num(model.depth_m * 1e3),
                  "problem_type": "axisymmetric" if model.problem_type == AXISYMMETRIC else "planar",
                  "frequency_hz": Num("0")},
        "nodes_mm": [[_num(x * 1e3), _num(y * 1e3)] for x, y in model.xy],
        "triangles": {"node_indices": [[Num(str(int(v))) for v in t] for t in model.tri],
                      "region_ids": [Num(str(int(m))) for m in model.tri_mat]},
        "regions": regions,
        "materials": mats,
        "circuits": [{"index": Num(str(c)), "name": f"c{c}", "type": "series",
                      "current_A": _num(currents[c])} for c in range(model.circuit_count)],
        "outer_dirichlet": {"node_indices": [Num(str(int(v))) for v in model.dir_nodes],
                            "A_Wb_per_m": [Num("0") for _ in model.dir_nodes]},
        "node_constraints": [{"node_a": Num(str(int(a))), "node_b": Num(str(int(b))),
                              "relation": "periodic" if s > 0 else "antiperiodic"}
                             for a, b, s in zip(model.con_a, model.con_b, model.con_sign)],
    }
    identity = canonical_sha256(resolved)
    root = {"schema_version": "gpu_femm_magnetostatic_mesh_v1", "source_fem_sha256": source_sha256,
            "canonical_identity_sha256": identity, "resolved": resolved}
    return _canonical(root), identity
