// artifact.cpp -- neutral mesh artifact parser (see artifact.h).
#include "artifact.h"

#include <cmath>
#include <map>

namespace fgio
{
namespace
{

constexpr double kMu0 = 4.0e-7 * 3.141592653589793238462643383279502884; // vacuum permeability

using K = Json::Kind;

// Twice the signed area of a triangle, in the order the library's element terms use.
double Det(const double *p0, const double *p1, const double *p2)
{
  return (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
}

} // namespace

fg_model Artifact::Model()
{
  curves.clear();
  for (size_t c = 0; c < curve_b.size(); ++c)
    curves.push_back(fg_bh_curve{static_cast<int32_t>(curve_b[c].size()), curve_b[c].data(),
                                 curve_h[c].data()});
  fg_model m{};
  m.problem_type = problem_type;
  m.node_count = static_cast<int32_t>(xy.size() / 2);
  m.node_xy = xy.data();
  m.triangle_count = static_cast<int32_t>(tri_mat.size());
  m.triangle_nodes = tri.data();
  m.triangle_material = tri_mat.data();
  m.material_count = static_cast<int32_t>(materials.size());
  m.materials = materials.data();
  m.curve_count = static_cast<int32_t>(curves.size());
  m.curves = curves.data();
  m.dirichlet_count = static_cast<int32_t>(dir_nodes.size());
  m.dirichlet_nodes = dir_nodes.data();
  m.dirichlet_values = dir_values.data();
  m.constraint_count = static_cast<int32_t>(con_signs.size());
  m.constraint_nodes = con_nodes.data();
  m.constraint_signs = con_signs.data();
  m.circuit_count = static_cast<int32_t>(circuit_currents.size());
  m.depth_m = depth_m;
  return m;
}

bool ParseArtifact(const std::string &text, Artifact *out, std::string *error)
{
  Json root;
  if (!ParseJson(text, &root, error))
    return false;
  const Json *schema = root.get("schema_version", K::String, error);
  if (!schema)
    return false;
  const bool planar_dc = schema->text == "gpu_femm_planar_dc_mesh_v1";
  const bool generic = schema->text == "gpu_femm_magnetostatic_mesh_v1";
  const bool neutral = planar_dc || generic;
  const bool motor = schema->text == "gpu_femm_mesh_v1";
  if (schema->text == "gpu_femm_mesh_v2" || schema->text == "gpu_femm_mesh_v3" ||
      schema->text == "gpu_femm_mesh_v4") {
    *error = "unsupported mesh artifact schema (native air-gap element and sector artifacts are not served "
             "here)";
    return false;
  }
  if (!neutral && !motor) {
    *error = "unsupported mesh artifact schema";
    return false;
  }
  if (!(neutral ? HasExactly(root, {"schema_version", "source_fem_sha256", "canonical_identity_sha256", "resolved"},
                             error)
                : HasExactly(root, {"schema_version", "base_motor_fem_sha256", "source_fem_sha256",
                                    "canonical_identity_sha256", "resolved"},
                             error)))
    return false;
  // Neutral schemas bind lower-case digests and the canonical identity; the motor schema
  // accepts any-case digests and carries no identity check (mesh_artifact.cpp:42-85).
  const bool lower = neutral;
  const Json *source = root.get("source_fem_sha256", K::String, error);
  const Json *root_base = neutral ? source : root.get("base_motor_fem_sha256", K::String, error);
  const Json *identity = root.get("canonical_identity_sha256", K::String, error);
  const Json *res = root.get("resolved", K::Object, error);
  const bool header_ok =
      source && root_base && identity && res && IsSha256Hex(root_base->text, lower) &&
      IsSha256Hex(source->text, lower) && IsSha256Hex(identity->text, lower) &&
      (generic ? HasExactly(*res, {"source_fem_sha256", "model", "nodes_mm", "triangles", "regions",
                                   "materials", "circuits", "outer_dirichlet", "node_constraints"}, error)
               : planar_dc ? HasExactly(*res, {"source_fem_sha256", "model", "nodes_mm", "triangles", "regions",
                                               "materials", "circuits", "outer_dirichlet"}, error)
                           : HasExactly(*res, {"source_fem_sha256", "base_motor_fem_sha256", "model", "pose",
                                               "nodes_mm", "triangles", "regions", "materials", "circuits",
                                               "outer_dirichlet"}, error));
  if (!header_ok) {
    if (error->empty())
      *error = "invalid GPU FEMM mesh artifact header";
    return false;
  }
  if (neutral && Sha256Hex(Canonical(*res)) != identity->text) {
    *error = "canonical artifact identity mismatch";
    return false;
  }
  const Json *rsource = res->get("source_fem_sha256", K::String, error);
  const Json *rbase = neutral ? rsource : res->get("base_motor_fem_sha256", K::String, error);
  const Json *model = res->get("model", K::Object, error);
  const Json *pose = neutral ? nullptr : res->get("pose", K::Object, error);
  const Json *nodes = res->get("nodes_mm", K::Array, error);
  const Json *triangles = res->get("triangles", K::Object, error);
  const Json *regions = res->get("regions", K::Array, error);
  const Json *materials = res->get("materials", K::Array, error);
  const Json *circuits = res->get("circuits", K::Array, error);
  const Json *boundary = res->get("outer_dirichlet", K::Object, error);
  const Json *constraints = generic ? res->get("node_constraints", K::Array, error) : nullptr;
  if (!rsource || !rbase || !model || (!neutral && !pose) || !nodes || !triangles || !regions || !materials ||
      !circuits || !boundary || (generic && !constraints) || !IsSha256Hex(rsource->text, lower) ||
      !IsSha256Hex(rbase->text, lower) || rsource->text != source->text || rbase->text != root_base->text) {
    if (error->empty())
      *error = "source FEM SHA mismatch";
    return false;
  }
  if (!HasExactly(*model, {"depth_mm", "problem_type", "frequency_hz"}, error))
    return false;
  const Json *depth = model->get("depth_mm", K::Number, error);
  const Json *type = model->get("problem_type", K::String, error);
  const Json *freq = model->get("frequency_hz", K::Number, error);
  const bool planar = type && type->text == "planar";
  const bool axi = type && type->text == "axisymmetric";
  if (!depth || !type || !freq || !(depth->number > 0.0) || freq->number != 0.0 || (!generic && !planar) ||
      (generic && !planar && !axi)) {
    *error = "unsupported model physics";
    return false;
  }
  const Json *rotor = nullptr, *displacement = nullptr;
  if (!neutral) {
    if (!HasExactly(*pose, {"rotor_angle_deg", "displacement_mm"}, error))
      return false;
    rotor = pose->get("rotor_angle_deg", K::Number, error);
    displacement = pose->get("displacement_mm", K::Array, error);
    if (!rotor || !displacement || displacement->items.size() != 2 || !displacement->items[0].is(K::Number) ||
        !displacement->items[1].is(K::Number)) {
      *error = "invalid pose";
      return false;
    }
  }
  if (nodes->items.size() < 3 || materials->items.empty() || regions->items.empty()) {
    *error = "empty mesh/material input";
    return false;
  }
  Artifact a;
  a.schema_version = schema->text;
  a.motor = motor;
  a.base_motor_fem_sha256 = root_base->text;
  a.rotor_angle_deg = motor ? rotor->number : 0.0;
  a.displacement_mm[0] = motor ? displacement->items[0].number : 0.0;
  a.displacement_mm[1] = motor ? displacement->items[1].number : 0.0;
  a.source_fem_sha256 = source->text;
  a.canonical_identity_sha256 = identity->text;
  a.problem_type = axi ? FG_AXISYMMETRIC : FG_PLANAR;
  a.depth_m = depth->number * 1e-3;
  for (const Json &p : nodes->items) {
    if (!p.is(K::Array) || p.items.size() != 2 || !p.items[0].is(K::Number) || !p.items[1].is(K::Number)) {
      *error = "invalid node coordinate";
      return false;
    }
    a.xy.push_back(p.items[0].number * 1e-3);
    a.xy.push_back(p.items[1].number * 1e-3);
  }
  const size_t N = a.xy.size() / 2;

  std::map<int32_t, int32_t> material_of;
  for (const Json &m : materials->items) {
    if (!HasExactly(m, {"id", "name", "mu_x", "mu_y", "H_c_A_per_m", "B_T", "H_A_per_m", "lam_type", "lam_fill"}, error))
      return false;
    const Json *id = m.get("id", K::Number, error);
    const Json *name = m.get("name", K::String, error);
    const Json *mux = m.get("mu_x", K::Number, error);
    const Json *muy = m.get("mu_y", K::Number, error);
    const Json *hc = m.get("H_c_A_per_m", K::Number, error);
    const Json *b = m.get("B_T", K::Array, error);
    const Json *h = m.get("H_A_per_m", K::Array, error);
    const Json *lam_type = m.get("lam_type", K::Number, error);
    const Json *lam_fill = m.get("lam_fill", K::Number, error);
    int32_t mid = -1;
    if (!id || !name || !mux || !muy || !hc || !b || !h || !lam_type || !lam_fill || !AsInt32(*id, &mid) ||
        mid < 0 || name->text.empty() || material_of.count(mid) || !(mux->number > 0.0) ||
        mux->number != muy->number || hc->number < 0.0 || lam_type->number != 0.0 ||
        lam_fill->number != 1.0 || b->items.size() != h->items.size()) {
      *error = "invalid material definition";
      return false;
    }
    fg_material mat{};
    mat.reluctivity_zero_m_per_h = 1.0 / (kMu0 * mux->number);
    mat.h_c_a_per_m = hc->number;
    mat.bh_curve_index = -1;
    mat.circuit_index = -1;
    mat.group_number = -1; // base materials carry no block-label group
    if (b->items.size() > 4096) {
      *error = "B-H curve exceeds point cap";
      return false;
    }
    if (!b->items.empty()) {
      if (b->items.size() < 2) {
        *error = "B-H curve needs two points";
        return false;
      }
      std::vector<double> bb, hh;
      for (size_t k = 0; k < b->items.size(); ++k) {
        const Json &bk = b->items[k], &hk = h->items[k];
        if (!bk.is(K::Number) || !hk.is(K::Number) || bk.number < 0.0 || hk.number < 0.0 ||
            (k > 0 && (bk.number < bb.back() || hk.number < hh.back()))) {
          *error = "invalid B-H point";
          return false;
        }
        bb.push_back(bk.number);
        hh.push_back(hk.number);
      }
      // The spline itself is built (and rejected if invalid) by fg_plan_create.
      mat.bh_curve_index = static_cast<int32_t>(a.curve_b.size());
      a.curve_b.push_back(std::move(bb));
      a.curve_h.push_back(std::move(hh));
    }
    material_of.emplace(mid, static_cast<int32_t>(a.materials.size()));
    a.materials.push_back(mat);
    a.group_numbers.push_back(-1);
  }
  for (size_t i = 0; i < circuits->items.size(); ++i) {
    const Json &c = circuits->items[i];
    if (!HasExactly(c, {"index", "name", "type", "current_A"}, error))
      return false;
    const Json *index = c.get("index", K::Number, error);
    const Json *name = c.get("name", K::String, error);
    const Json *ctype = c.get("type", K::String, error);
    const Json *current = c.get("current_A", K::Number, error);
    int32_t ci = -1;
    if (!index || !name || !ctype || !current || !AsInt32(*index, &ci) || ci != static_cast<int32_t>(i) ||
        name->text.empty() || ctype->text != "series") {
      *error = "circuits must be ordered contiguous current-driven series circuits";
      return false;
    }
    a.circuit_currents.push_back(current->number);
  }
  const int32_t C = static_cast<int32_t>(a.circuit_currents.size());
  struct Region {
    int32_t material, circuit, group;
    double turns, angle;
  };
  std::vector<Region> regs;
  std::map<int32_t, int32_t> region_of;
  for (const Json &r : regions->items) {
    if (!HasExactly(r, {"id", "group_number", "material_id", "circuit_index", "turns", "pm_magnetization_deg"}, error))
      return false;
    const Json *id = r.get("id", K::Number, error);
    const Json *group = r.get("group_number", K::Number, error);
    const Json *mat = r.get("material_id", K::Number, error);
    const Json *circ = r.get("circuit_index", K::Number, error);
    const Json *turns = r.get("turns", K::Number, error);
    const Json *angle = r.get("pm_magnetization_deg", K::Number, error);
    int32_t rid = -1, gid = -1, mid = -1, cid = -2;
    if (!id || !group || !mat || !circ || !turns || !angle || !AsInt32(*id, &rid) || !AsInt32(*group, &gid) ||
        !AsInt32(*mat, &mid) || !AsInt32(*circ, &cid) || rid < 0 || gid < 0 || !material_of.count(mid) ||
        region_of.count(rid) || cid < -1 || (cid == -1 && turns->number != 0.0) ||
        (cid >= 0 && (cid >= C || turns->number == 0.0))) {
      *error = "invalid region definition";
      return false;
    }
    region_of.emplace(rid, static_cast<int32_t>(regs.size()));
    regs.push_back({material_of[mid], cid, gid, turns->number, angle->number});
  }
  if (!HasExactly(*triangles, {"node_indices", "region_ids"}, error))
    return false;
  const Json *faces = triangles->get("node_indices", K::Array, error);
  const Json *fregions = triangles->get("region_ids", K::Array, error);
  if (!faces || !fregions || faces->items.empty() || faces->items.size() != fregions->items.size()) {
    *error = "invalid triangle arrays";
    return false;
  }
  std::vector<double> area(regs.size(), 0.0);
  std::vector<int32_t> treg;
  for (size_t e = 0; e < faces->items.size(); ++e) {
    const Json &f = faces->items[e];
    if (!f.is(K::Array) || f.items.size() != 3) {
      *error = "triangle must have three node indices";
      return false;
    }
    int32_t rid = -1, v[3];
    if (!fregions->items[e].is(K::Number) || !AsInt32(fregions->items[e], &rid) || !region_of.count(rid)) {
      *error = "triangle references unknown region";
      return false;
    }
    for (int l = 0; l < 3; ++l)
      if (!AsInt32(f.items[l], &v[l]) || v[l] < 0 || static_cast<size_t>(v[l]) >= N) {
        *error = "triangle node out of range";
        return false;
      }
    const double det = Det(&a.xy[2 * v[0]], &a.xy[2 * v[1]], &a.xy[2 * v[2]]);
    if (!(det > 0.0) || !std::isfinite(det)) {
      *error = "triangle is not CCW";
      return false;
    }
    const int32_t k = region_of[rid];
    area[k] += 0.5 * det;
    a.tri.insert(a.tri.end(), v, v + 3);
    treg.push_back(k);
  }
  const int32_t labels = static_cast<int32_t>(a.materials.size());
  for (size_t k = 0; k < regs.size(); ++k) {
    if (!(area[k] > 0.0)) {
      *error = "region has no triangle area";
      return false;
    }
    fg_material label = a.materials[regs[k].material];
    label.group_number = regs[k].group;
    label.circuit_index = regs[k].circuit;
    label.magnetization_deg = regs[k].angle;
    label.source_j_per_a = regs[k].circuit < 0 ? 0.0 : regs[k].turns / area[k];
    a.materials.push_back(label);
    a.group_numbers.push_back(regs[k].group);
  }
  for (int32_t k : treg)
    a.tri_mat.push_back(labels + k);
  if (!HasExactly(*boundary, {"node_indices", "A_Wb_per_m"}, error))
    return false;
  const Json *bn = boundary->get("node_indices", K::Array, error);
  const Json *bv = boundary->get("A_Wb_per_m", K::Array, error);
  if (!bn || !bv || bn->items.empty() || bn->items.size() != bv->items.size()) {
    *error = "invalid outer Dirichlet";
    return false;
  }
  for (size_t i = 0; i < bn->items.size(); ++i) {
    int32_t node = -1;
    if (!AsInt32(bn->items[i], &node) || node < 0 || static_cast<size_t>(node) >= N ||
        !bv->items[i].is(K::Number) || bv->items[i].number != 0.0) {
      *error = "outer Dirichlet must be zero and in range";
      return false;
    }
    a.dir_nodes.push_back(node);
    a.dir_values.push_back(0.0);
  }
  if (generic) {
    for (const Json &c : constraints->items) {
      if (!HasExactly(c, {"node_a", "node_b", "relation"}, error))
        return false;
      const Json *na = c.get("node_a", K::Number, error);
      const Json *nb = c.get("node_b", K::Number, error);
      const Json *rel = c.get("relation", K::String, error);
      int32_t ia = -1, ib = -1;
      if (!na || !nb || !rel || !AsInt32(*na, &ia) || !AsInt32(*nb, &ib) || ia < 0 || ib < 0 ||
          static_cast<size_t>(ia) >= N || static_cast<size_t>(ib) >= N || ia == ib ||
          (rel->text != "periodic" && rel->text != "antiperiodic")) {
        *error = "invalid periodic node constraint";
        return false;
      }
      a.con_nodes.push_back(ia);
      a.con_nodes.push_back(ib);
      a.con_signs.push_back(rel->text == "periodic" ? 1 : -1);
    }
  }
  *out = std::move(a);
  return true;
}

} // namespace fgio
