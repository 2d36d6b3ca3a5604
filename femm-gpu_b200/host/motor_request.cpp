// motor_request.cpp -- motor sample requests and the motor batch envelope.
#include "motor_request.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <set>

namespace fgio
{
namespace
{

using K = Json::Kind;

// An array of numbers (StrictNumberArray, sample_request.cpp:138-151).
bool Numbers(const Json &v, std::vector<double> *out)
{
  if (!v.is(K::Array))
    return false;
  out->clear();
  for (const Json &x : v.items) {
    if (!x.is(K::Number))
      return false;
    out->push_back(x.number);
  }
  return true;
}

bool Identifier(const std::string &s, size_t max_len)
{
  return !s.empty() && s.size() <= max_len && std::all_of(s.begin(), s.end(), [](unsigned char c) {
    return std::isalnum(c) || c == '_' || c == '-' || c == '.';
  });
}

} // namespace

bool ParseMotorSampleRequest(const Json &root, MotorSampleRequest *r, std::string *error)
{
  std::string version;
  if (root.is(K::Object)) {
    auto it = root.members.find("protocol");
    if (it != root.members.end() && it->second.is(K::String))
      version = it->second.text;
  }
  const bool v1 = version == "gpu_femm_motor_sample_v1", v2 = version == "gpu_femm_motor_sample_v2";
  const bool v3 = version == "gpu_femm_motor_sample_v3", v4 = version == "gpu_femm_motor_sample_v4";
  const bool has_tangent = root.is(K::Object) && root.members.count("tangent_multi_rhs") != 0;
  if ((!v1 && !v2 && !v3 && !v4) ||
      (v1 && !HasExactly(root, {"protocol", "mesh_artifact_path", "mesh_artifact_sha256", "base_motor_fem_sha256",
                                "source_fem_sha256", "circuit_currents_A", "selected_group_number",
                                "air_group_number", "airgap_radius_mm", "airgap_angles_deg",
                                "rotor_angle_deg", "displacement_mm"},
                         error)) ||
      (v2 && !has_tangent) ||
      (v2 && !HasExactly(root, {"protocol", "mesh_artifact_path", "mesh_artifact_sha256", "base_motor_fem_sha256",
                                "source_fem_sha256", "circuit_currents_A", "selected_group_number",
                                "air_group_number", "airgap_radius_mm", "airgap_angles_deg",
                                "rotor_angle_deg", "displacement_mm", "tangent_multi_rhs"},
                         error)) ||
      ((v3 || v4) && !HasExactly(root, {"protocol", "mesh_artifact_path", "mesh_artifact_sha256",
                                        "base_motor_fem_sha256", "source_fem_sha256", "circuit_currents_A",
                                        "selected_group_number", "air_group_number", "airgap_radius_mm",
                                        "airgap_angles_deg", "rotor_angle_deg", "displacement_mm",
                                        "tangent_multi_rhs", "sector_performance"},
                                 error)))
    return false;
  const Json *protocol = root.get("protocol", K::String, error);
  const Json *path = root.get("mesh_artifact_path", K::String, error);
  const Json *artifact_sha = root.get("mesh_artifact_sha256", K::String, error);
  const Json *base_sha = root.get("base_motor_fem_sha256", K::String, error);
  const Json *source_sha = root.get("source_fem_sha256", K::String, error);
  const Json *currents = root.get("circuit_currents_A", K::Array, error);
  const Json *selected = root.get("selected_group_number", K::Number, error);
  const Json *air = root.get("air_group_number", K::Number, error);
  const Json *radius = root.get("airgap_radius_mm", K::Number, error);
  const Json *angles = root.get("airgap_angles_deg", K::Array, error);
  const Json *rotor = root.get("rotor_angle_deg", K::Number, error);
  const Json *displacement = root.get("displacement_mm", K::Array, error);
  int32_t sel = -1, airg = -1;
  if (!protocol || !path || !artifact_sha || !base_sha || !source_sha || !currents || !selected || !air ||
      !radius || !angles || !rotor || !displacement || path->text.empty() || !IsSha256Hex(artifact_sha->text, false) ||
      !IsSha256Hex(base_sha->text, false) || !IsSha256Hex(source_sha->text, false) || !AsInt32(*selected, &sel) ||
      !AsInt32(*air, &airg) || sel < 0 || airg < 0 || sel == airg || !(radius->number >= 0.0) ||
      displacement->items.size() != 2 || !displacement->items[0].is(K::Number) ||
      !displacement->items[1].is(K::Number) || !Numbers(*currents, &r->circuit_currents_a) ||
      !Numbers(*angles, &r->airgap_angles_deg) || r->circuit_currents_a.empty() ||
      (!r->airgap_angles_deg.empty() && !(radius->number > 0.0))) {
    if (error->empty())
      *error = "invalid gpu_femm_motor_sample_v1 request";
    return false;
  }
  r->protocol = protocol->text;
  r->mesh_artifact_path = path->text;
  r->mesh_artifact_sha256 = artifact_sha->text;
  r->base_motor_fem_sha256 = base_sha->text;
  r->source_fem_sha256 = source_sha->text;
  r->selected_group_number = sel;
  r->air_group_number = airg;
  r->airgap_radius_mm = radius->number;
  r->rotor_angle_deg = rotor->number;
  r->displacement_mm[0] = displacement->items[0].number;
  r->displacement_mm[1] = displacement->items[1].number;
  r->tangent_requested = false;
  r->tangent_rhs.clear();
  r->sector_performance = false;
  r->model_invariance_certificate_sha256.clear();
  if (v2 || v3 || v4) {
    const Json &tangent = root.members.at("tangent_multi_rhs");
    // An unused nested struct arrives as null or [] from MATLAB encoders: no tangent.
    const bool empty = tangent.is(K::Null) || (tangent.is(K::Array) && tangent.items.empty());
    if (empty && v2)
      return true;
    if (!empty) {
      if (!HasExactly(tangent, {"schema_version", "rhs"}, error))
        return false;
      const Json *schema = tangent.get("schema_version", K::String, error);
      const Json *rhs = tangent.get("rhs", K::Array, error);
      if (!schema || !rhs || schema->text != "gpu_femm_tangent_multi_rhs_v1" || rhs->items.empty() ||
          rhs->items.size() > 8) {
        if (error->empty())
          *error = "invalid gpu_femm_tangent_multi_rhs_v1 request";
        return false;
      }
      std::set<std::string> names;
      for (const Json &entry : rhs->items) {
        if (!HasExactly(entry, {"name", "circuit_current_derivative_A_per_A"}, error))
          return false;
        const Json *name = entry.get("name", K::String, error);
        const Json *dir = entry.get("circuit_current_derivative_A_per_A", K::Array, error);
        std::vector<double> values;
        if (!name || !Identifier(name->text, 128) || !dir || names.count(name->text) ||
            !Numbers(*dir, &values) || values.size() != r->circuit_currents_a.size() ||
            !std::all_of(values.begin(), values.end(), [](double v) { return std::isfinite(v); })) {
          if (error->empty())
            *error = "invalid tangent RHS name or circuit derivative vector";
          return false;
        }
        names.insert(name->text);
        r->tangent_rhs.emplace_back(name->text, std::move(values));
      }
      r->tangent_requested = true;
    }
  }
  if (v3 || v4) {
    const Json &sector = root.members.at("sector_performance");
    if (!HasExactly(sector, {"schema_version", "model_invariance_certificate_sha256"}, error))
      return false;
    const Json *schema = sector.get("schema_version", K::String, error);
    const Json *cert = sector.get("model_invariance_certificate_sha256", K::String, error);
    if (!schema || !cert || !IsSha256Hex(cert->text) ||
        schema->text != (v4 ? "gpu_femm_motor_sector_performance_v2" : "gpu_femm_motor_sector_performance_v1")) {
      *error = "invalid gpu_femm_motor_sector_performance_v1 request";
      return false;
    }
    r->sector_performance = true;
    r->model_invariance_certificate_sha256 = cert->text;
  }
  if (v4 && r->tangent_requested) {
    *error = "gpu_femm_motor_sample_v4 rejects tangent_multi_rhs";
    return false;
  }
  return true;
}

bool ParseMotorSampleRequestText(const std::string &text, MotorSampleRequest *out, std::string *error)
{
  Json root;
  return ParseJson(text, &root, error) && ParseMotorSampleRequest(root, out, error);
}

bool MotorRequestMatchesArtifact(const MotorSampleRequest &r, const Artifact &a)
{
  // Neutral artifacts carry their source digest as the base identity and a zero pose; v3
  // requests take conforming sectors, v4 requests native air-gap element sectors.
  const bool sector_request = r.protocol == "gpu_femm_motor_sample_v3";
  const bool native_request = r.protocol == "gpu_femm_motor_sample_v4";
  if (sector_request != (a.sector && !a.native_sector) || native_request != a.native_sector)
    return false;
  if (native_request &&
      (a.schema_version != "gpu_femm_mesh_v4" || a.full_machine_sector_count < 2 ||
       a.sector_angle_deg != 360.0 / a.full_machine_sector_count || !a.sliding_band || a.bands.empty() ||
       !r.sector_performance || r.model_invariance_certificate_sha256 != a.model_invariance_certificate_sha256))
    return false;
  if (sector_request &&
      (a.schema_version != "gpu_femm_mesh_v3" || a.sector_angle_deg != 180.0 || a.full_machine_sector_count != 2 ||
       a.electrical_pole_pairs <= 0 || a.suspension_spatial_order != a.electrical_pole_pairs + 1 ||
       a.sector_boundary_sign != (a.electrical_pole_pairs % 2 == 0 ? 1 : -1) || !r.sector_performance ||
       r.model_invariance_certificate_sha256 != a.model_invariance_certificate_sha256))
    return false;
  // A sliding-band artifact serves any rotor angle at zero displacement; its postprocess
  // groups must exist and the probe circle must lie in every band (sample_request.cpp:
  // 413-438).  A conforming artifact is one pose.
  bool pose = false, post = true;
  if (a.sliding_band) {
    pose = r.displacement_mm[0] == 0.0 && r.displacement_mm[1] == 0.0;
    auto has_group = [&a](int32_t g) { return std::find(a.group_numbers.begin(), a.group_numbers.end(), g) != a.group_numbers.end(); };
    post = has_group(r.selected_group_number) && has_group(r.air_group_number);
    if (post && !r.airgap_angles_deg.empty()) {
      post = !a.bands.empty();
      for (const AirGapBand &b : a.bands) {
        const double ri = 1000.0 * b.ri_m, ro = 1000.0 * b.ro_m, tol = 1e-9 * std::max(1.0, std::abs(ro));
        post = post && r.airgap_radius_mm >= ri - tol && r.airgap_radius_mm <= ro + tol;
      }
    }
  } else {
    pose = r.rotor_angle_deg == a.rotor_angle_deg && r.displacement_mm[0] == a.displacement_mm[0] &&
           r.displacement_mm[1] == a.displacement_mm[1];
  }
  return r.base_motor_fem_sha256 == a.base_motor_fem_sha256 && r.source_fem_sha256 == a.source_fem_sha256 &&
         pose && post && r.circuit_currents_a.size() == a.circuit_currents.size();
}

bool ParseMotorBatchRequestText(const std::string &text, MotorBatchRequest *b, std::string *error)
{
  Json root;
  if (!ParseJson(text, &root, error) || !HasExactly(root, {"protocol", "max_items_per_chunk", "items"}, error))
    return false;
  const Json *protocol = root.get("protocol", K::String, error);
  const Json *chunk = root.get("max_items_per_chunk", K::Number, error);
  const Json *items = root.get("items", K::Array, error);
  int32_t width = 0;
  if (!protocol || !chunk || !items ||
      (protocol->text != "gpu_femm_motor_batch_v1" && protocol->text != "gpu_femm_motor_batch_v2" &&
       protocol->text != "gpu_femm_motor_batch_v3" && protocol->text != "gpu_femm_motor_batch_v4") ||
      !AsInt32(*chunk, &width) || width < 1 || width > 4096 || items->items.empty() || items->items.size() > 4096) {
    if (error->empty())
      *error = "invalid gpu_femm_motor_batch_v1 request";
    return false;
  }
  b->protocol = protocol->text;
  b->max_items_per_chunk = width;
  b->items.clear();
  // The item protocol must be the sample version of the batch version.
  const std::string expected = "gpu_femm_motor_sample_v" + protocol->text.substr(protocol->text.size() - 1);
  std::set<std::string> ids;
  for (const Json &item : items->items) {
    if (!HasExactly(item, {"task_id", "request"}, error))
      return false;
    const Json *id = item.get("task_id", K::String, error);
    const Json *sample = item.get("request", K::Object, error);
    MotorBatchItem parsed;
    if (!id || !sample || !Identifier(id->text, 256) || ids.count(id->text) ||
        !ParseMotorSampleRequest(*sample, &parsed.request, error)) {
      if (error->empty())
        *error = "invalid or duplicate batch task_id";
      return false;
    }
    if (parsed.request.protocol != expected) {
      *error = "motor batch and item protocol versions must match";
      return false;
    }
    parsed.task_id = id->text;
    ids.insert(parsed.task_id);
    b->items.push_back(std::move(parsed));
  }
  return true;
}

} // namespace fgio
