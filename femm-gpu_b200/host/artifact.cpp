// artifact.cpp -- neutral mesh artifact parser (see artifact.h).
#include "artifact.h"

#include <algorithm>
#include <cmath>
#include <limits>
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
  band_view.clear();
  for (const AirGapBand &b : bands) {
    fg_air_gap_element e{};
    e.antiperiodic = b.antiperiodic ? 1 : 0;
    e.point_count = static_cast<int32_t>(b.nodes.size() / 4);
    e.center_x_m = b.center_m[0];
    e.center_y_m = b.center_m[1];
    e.inner_radius_m = b.ri_m;
    e.outer_radius_m = b.ro_m;
    e.arc_length_deg = b.arc_deg;
    e.inner_shift = b.inner_shift;
    e.outer_shift = b.outer_shift;
    e.nodes = b.nodes.data();
    e.weights = b.weights.data();
    band_view.push_back(e);
  }
  m.air_gap_count = static_cast<int32_t>(band_view.size());
  m.air_gap_elements = band_view.empty() ? nullptr : band_view.data();
  return m;
}

bool Artifact::SlideBands(double rotor_angle_deg)
{
  if (!sliding_band)
    return true;
  const double delta = rotor_angle_deg - this->rotor_angle_deg;
  if (!std::isfinite(delta))
    return false;
  for (AirGapBand &b : bands) {
    const int64_t arcs = static_cast<int64_t>(b.nodes.size() / 4) - 1;
    if (arcs <= 0 || !(b.arc_deg > 0.0))
      return false;
    const double slid = b.inner_shift + delta * static_cast<double>(arcs) / b.arc_deg;
    const int64_t whole = static_cast<int64_t>(std::floor(slid));
    b.inner_shift = slid - static_cast<double>(whole);
    const std::vector<int32_t> nodes = b.nodes;
    const std::vector<double> weights = b.weights;
    for (int64_t k = 0; k < arcs; ++k) {
      int64_t from = (k - whole) % arcs;
      if (from < 0)
        from += arcs;
      for (int l = 0; l < 2; ++l) {
        b.nodes[4 * k + l] = nodes[4 * from + l];
        b.weights[4 * k + l] = weights[4 * from + l];
      }
    }
    for (int l = 0; l < 2; ++l) {
      b.nodes[4 * arcs + l] = b.nodes[l];
      b.weights[4 * arcs + l] = b.weights[l];
    }
  }
  return true;
}

// The sector metadata of gpu_femm_mesh_v3 / v4 (mesh_artifact.cpp:441-608): p pole pairs,
// the p + 1 suspension order, the boundary relation of the pole-pair parity, apex
// self-pairs at the origin, a circuit partner map that closes after k copies with positive
// orientation.  v3 (conforming) is the 180-degree half with every constraint pair related
// by an exact 180-degree rotation; v4 (native air-gap element, `native`) is one of k
// sectors of 360/k degrees whose electrical phase advance 2p/k is an integer, odd exactly
// for an antiperiodic relation, every pair related by the sector rotation either way.  An
// antiperiodic sector fixes its apex nodes to zero.
bool ParseSector(const Json &sec, bool native, Artifact *a, std::string *error)
{
  if (!HasExactly(sec, {"schema_version", "sector_start_angle_deg", "angle_deg", "full_machine_sector_count",
                        "electrical_pole_pairs", "suspension_spatial_order", "boundary_relation",
                        "circuit_partner_indices", "circuit_partner_orientations", "apex_self_pair_nodes",
                        "model_invariance_certificate_sha256"},
                  error))
    return false;
  const Json *schema = sec.get("schema_version", K::String, error);
  const Json *start = sec.get("sector_start_angle_deg", K::Number, error);
  const Json *angle = sec.get("angle_deg", K::Number, error);
  const Json *repeats = sec.get("full_machine_sector_count", K::Number, error);
  const Json *pole_pairs = sec.get("electrical_pole_pairs", K::Number, error);
  const Json *order = sec.get("suspension_spatial_order", K::Number, error);
  const Json *relation = sec.get("boundary_relation", K::String, error);
  const Json *partners = sec.get("circuit_partner_indices", K::Array, error);
  const Json *orientations = sec.get("circuit_partner_orientations", K::Array, error);
  const Json *apex = sec.get("apex_self_pair_nodes", K::Array, error);
  const Json *cert = sec.get("model_invariance_certificate_sha256", K::String, error);
  int32_t k = 0, p = 0, n = 0;
  const size_t C = a->circuit_currents.size();
  if (!schema || !start || !std::isfinite(start->number) || !angle || !repeats || !pole_pairs || !order ||
      !relation || !partners || !orientations || !apex || !cert || !IsSha256Hex(cert->text) ||
      schema->text != (native ? "gpu_femm_motor_sector_v2" : "gpu_femm_motor_sector_v1") ||
      !(angle->number > 0.0) || !AsInt32(*repeats, &k) || k < 2 ||
      !AsInt32(*pole_pairs, &p) || p <= 0 || !AsInt32(*order, &n) || n != p + 1 ||
      (relation->text != "periodic" && relation->text != "antiperiodic") || partners->items.size() != C ||
      orientations->items.size() != C) {
    *error = "motor sector requires positive k, p and p+1 harmonic metadata";
    return false;
  }
  if ((!native && (angle->number != 180.0 || k != 2)) || (native && angle->number != 360.0 / static_cast<double>(k))) {
    *error = "motor sector angle/count are inconsistent";
    return false;
  }
  if (native && ((2 * p) % k != 0 || (relation->text == "antiperiodic") != (((2 * p / k) % 2) != 0))) {
    *error = "native AGE sector boundary relation does not match electrical phase advance";
    return false;
  }
  a->sector = true;
  a->sector_start_angle_deg = start->number;
  a->sector_angle_deg = angle->number;
  a->full_machine_sector_count = k;
  a->electrical_pole_pairs = p;
  a->suspension_spatial_order = n;
  a->sector_boundary_sign = relation->text == "periodic" ? 1 : -1;
  a->model_invariance_certificate_sha256 = cert->text;
  const size_t N = a->xy.size() / 2;
  double radius = 1e-3;
  for (size_t i = 0; i < N; ++i)
    radius = std::max(radius, std::hypot(a->xy[2 * i], a->xy[2 * i + 1]));
  const double tol = std::max(1e-10 * radius, 64.0 * std::numeric_limits<double>::epsilon() * radius);
  const double turn = angle->number * 3.141592653589793238462643383279502884 / 180.0;
  const double cs = std::cos(turn), sn = std::sin(turn);
  for (size_t c = 0; c < a->con_signs.size(); ++c) {
    const double *pa = &a->xy[2 * a->con_nodes[2 * c]], *pb = &a->xy[2 * a->con_nodes[2 * c + 1]];
    if (!native && std::hypot(pa[0] + pb[0], pa[1] + pb[1]) > tol) {
      *error = "motor sector non-self constraint nodes must be related by an exact 180-degree rotation";
      return false;
    }
    // v4: either node may be the rotated one (the wire order is not the generator's).
    if (native && std::min(std::hypot(pb[0] - (cs * pa[0] - sn * pa[1]), pb[1] - (sn * pa[0] + cs * pa[1])),
                           std::hypot(pa[0] - (cs * pb[0] - sn * pb[1]), pa[1] - (sn * pb[0] + cs * pb[1]))) > tol) {
      *error = "motor sector non-self constraint nodes must be related by the sector rotation";
      return false;
    }
  }
  std::vector<bool> seen(N, false);
  for (const Json &x : apex->items) {
    int32_t node = -1;
    bool bad = !AsInt32(x, &node) || node < 0 || static_cast<size_t>(node) >= N;
    bad = bad || seen[node] || std::hypot(a->xy[2 * node], a->xy[2 * node + 1]) > tol;
    for (size_t c = 0; !bad && c < a->con_nodes.size(); ++c)
      bad = a->con_nodes[c] == node;
    bad = bad || std::find(a->dir_nodes.begin(), a->dir_nodes.end(), node) != a->dir_nodes.end();
    if (bad) {
      *error = "motor sector apex self-pair nodes must be unique origin nodes separate from physical boundaries "
               "and non-self constraints";
      return false;
    }
    seen[node] = true;
    a->apex_nodes.push_back(node);
  }
  std::vector<bool> used(C, false);
  for (size_t c = 0; c < C; ++c) {
    int32_t partner = -1, orientation = 0;
    if (!AsInt32(partners->items[c], &partner) || !AsInt32(orientations->items[c], &orientation) || partner < 0 ||
        static_cast<size_t>(partner) >= C || used[partner] || (orientation != -1 && orientation != 1)) {
      *error = "invalid motor sector circuit partner mapping";
      return false;
    }
    used[partner] = true;
    a->circuit_partners.push_back(partner);
    a->circuit_orientations.push_back(static_cast<int8_t>(orientation));
  }
  for (size_t c = 0; c < C; ++c) {
    int32_t at = static_cast<int32_t>(c);
    int sign = 1;
    for (int32_t copy = 0; copy < k; ++copy) {
      sign *= a->circuit_orientations[at];
      at = a->circuit_partners[at];
    }
    if (at != static_cast<int32_t>(c) || sign != 1) {
      *error = "motor sector circuit generator must close after k copies with positive orientation";
      return false;
    }
  }
  if (a->con_signs.empty() ||
      !std::all_of(a->con_signs.begin(), a->con_signs.end(), [&](int8_t s) { return s == a->sector_boundary_sign; })) {
    *error = "motor sector node constraints do not match boundary_relation";
    return false;
  }
  const int base_sign = p % 2 == 0 ? 1 : -1;
  if (a->sector_boundary_sign != base_sign) {
    *error = "motor sector boundary_relation does not match electrical pole-pair parity";
    return false;
  }
  if (base_sign < 0)
    for (int32_t node : a->apex_nodes) {
      a->dir_nodes.push_back(node);
      a->dir_values.push_back(0.0);
    }
  return true;
}

// The air_gap_elements of gpu_femm_mesh_v2 (mesh_artifact.cpp:609-697): a centred,
// zero-degree reference pose; one element object or a nonempty array of them, each with
// exactly its ten members, sector_count >= 2 arcs and sector_count + 1 points of integer
// nodes and numeric weights; every node in range (ValidateNonlinearModel's check).
bool ParseBands(const Json &res, Artifact *a, std::string *error)
{
  const auto it = res.members.find("air_gap_elements");
  if (it == res.members.end() || (!it->second.is(K::Array) && !it->second.is(K::Object)) ||
      a->displacement_mm[0] != 0.0 || a->displacement_mm[1] != 0.0 || a->rotor_angle_deg != 0.0) {
    *error = "sliding-band artifacts require a centered zero-degree reference mesh";
    return false;
  }
  std::vector<const Json *> entries;
  if (it->second.is(K::Array)) {
    if (it->second.items.empty()) {
      *error = "sliding-band requires an air-gap element";
      return false;
    }
    for (const Json &e : it->second.items)
      entries.push_back(&e);
  } else {
    entries.push_back(&it->second);
  }
  const size_t N = a->xy.size() / 2;
  for (const Json *e : entries) {
    if (!HasExactly(*e, {"name", "periodicity", "center_mm", "ri_mm", "ro_mm", "arc_length_deg", "sector_count",
                         "inner_shift", "outer_shift", "quad_points"},
                    error))
      return false;
    const Json *name = e->get("name", K::String, error);
    const Json *per = e->get("periodicity", K::String, error);
    const Json *center = e->get("center_mm", K::Array, error);
    const Json *ri = e->get("ri_mm", K::Number, error);
    const Json *ro = e->get("ro_mm", K::Number, error);
    const Json *arc = e->get("arc_length_deg", K::Number, error);
    const Json *sectors = e->get("sector_count", K::Number, error);
    const Json *ishift = e->get("inner_shift", K::Number, error);
    const Json *oshift = e->get("outer_shift", K::Number, error);
    const Json *points = e->get("quad_points", K::Array, error);
    int32_t count = 0;
    if (!name || name->text.empty() || !per || !center || !ri || !ro || !arc || !sectors || !ishift || !oshift ||
        !points || center->items.size() != 2 || !center->items[0].is(K::Number) ||
        !center->items[1].is(K::Number) || !AsInt32(*sectors, &count) || count < 2 ||
        points->items.size() != static_cast<size_t>(count) + 1 ||
        (per->text != "periodic" && per->text != "antiperiodic")) {
      *error = "invalid sliding-band air-gap element";
      return false;
    }
    AirGapBand b;
    b.name = name->text;
    b.antiperiodic = per->text == "antiperiodic";
    b.center_m[0] = center->items[0].number * 1e-3;
    b.center_m[1] = center->items[1].number * 1e-3;
    b.ri_m = ri->number * 1e-3;
    b.ro_m = ro->number * 1e-3;
    b.arc_deg = arc->number;
    b.sector_count = count;
    b.inner_shift = ishift->number;
    b.outer_shift = oshift->number;
    for (const Json &pt : points->items) {
      if (!HasExactly(pt, {"n0", "w0", "n1", "w1", "n2", "w2", "n3", "w3"}, error))
        return false;
      for (int l = 0; l < 4; ++l) {
        const std::string nn = std::string("n") + char('0' + l), wn = std::string("w") + char('0' + l);
        const Json *node = pt.get(nn.c_str(), K::Number, error);
        const Json *weight = pt.get(wn.c_str(), K::Number, error);
        int32_t id = -1;
        if (!node || !weight || !AsInt32(*node, &id)) {
          *error = "invalid sliding-band quadrature point";
          return false;
        }
        b.nodes.push_back(id);
        b.weights.push_back(weight->number);
      }
    }
    a->bands.push_back(std::move(b));
  }
  for (const AirGapBand &b : a->bands)
    for (size_t l = 0; l < b.nodes.size(); ++l)
      if (b.nodes[l] < 0 || static_cast<size_t>(b.nodes[l]) >= N || !std::isfinite(b.weights[l]) ||
          !(b.ri_m > 0.0) || !(b.ro_m > b.ri_m) || !(b.arc_deg > 0.0) || !std::isfinite(b.inner_shift) ||
          !std::isfinite(b.outer_shift)) {
        *error = "mapped mesh model validation failed";
        return false;
      }
  a->sliding_band = true;
  return true;
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
  const bool motor_v1 = schema->text == "gpu_femm_mesh_v1";
  const bool native = schema->text == "gpu_femm_mesh_v4"; // a native air-gap element sector
  const bool sliding = schema->text == "gpu_femm_mesh_v2" || native;
  const bool sector = schema->text == "gpu_femm_mesh_v3" || native;
  const bool motor = motor_v1 || sliding || sector;
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
               : motor_v1 ? HasExactly(*res, {"source_fem_sha256", "base_motor_fem_sha256", "model", "pose",
                                              "nodes_mm", "triangles", "regions", "materials", "circuits",
                                              "outer_dirichlet"}, error)
               : (sliding && !native) ? HasExactly(*res, {"source_fem_sha256", "base_motor_fem_sha256", "model", "pose",
                                             "nodes_mm", "triangles", "regions", "materials", "circuits",
                                             "outer_dirichlet", "air_gap_elements"}, error)
                          : HasExactly(*res, {"source_fem_sha256", "base_motor_fem_sha256", "model", "pose",
                                              "nodes_mm", "triangles", "regions", "materials", "circuits",
                                              "outer_dirichlet", "air_gap_elements", "node_constraints",
                                              "sector"}, error));
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
  const Json *constraints = (generic || sector) ? res->get("node_constraints", K::Array, error) : nullptr;
  const Json *sector_meta = sector ? res->get("sector", K::Object, error) : nullptr;
  if (!rsource || !rbase || !model || (!neutral && !pose) || !nodes || !triangles || !regions || !materials ||
      !circuits || !boundary || ((generic || sector) && !constraints) || (sector && !sector_meta) ||
      !IsSha256Hex(rsource->text, lower) ||
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
  if (sector && !native) {
    // gpu_femm_mesh_v3 is a conforming posed sector: its air-gap element list must be empty.
    const auto ages = res->members.find("air_gap_elements");
    if (ages == res->members.end() || !ages->second.is(K::Array) || !ages->second.items.empty()) {
      *error = "gpu_femm_mesh_v3 requires a conforming posed sector mesh; native AGE sectors are not supported";
      return false;
    }
  }
  if (native) {
    const auto ages = res->members.find("air_gap_elements");
    if (ages == res->members.end() || (!ages->second.is(K::Array) && !ages->second.is(K::Object)) ||
        (ages->second.is(K::Array) && ages->second.items.empty())) {
      *error = "gpu_femm_mesh_v4 requires a nonempty native AGE sector";
      return false;
    }
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
  if (generic || sector) {
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
  if (sector && !ParseSector(*sector_meta, native, &a, error))
    return false;
  if (sliding && !ParseBands(*res, &a, error))
    return false;
  if (native) {
    a.native_sector = true;
    for (const AirGapBand &b : a.bands)
      if (b.antiperiodic != (a.sector_boundary_sign < 0) || b.arc_deg != a.sector_angle_deg) {
        *error = "native AGE sector periodicity or arc length disagrees with sector metadata";
        return false;
      }
  }
  *out = std::move(a);
  return true;
}

} // namespace fgio
