// request.cpp -- sample request and batch envelope parsing (see request.h).
#include "request.h"

#include <cctype>
#include <set>

namespace fgio
{
namespace
{

using K = Json::Kind;

bool NumberArray(const Json &a, std::vector<double> *out)
{
  out->clear();
  for (const Json &v : a.items) {
    if (!v.is(K::Number))
      return false;
    out->push_back(v.number);
  }
  return true;
}

bool TaskIdValid(const std::string &id)
{
  if (id.empty() || id.size() > 256)
    return false;
  for (unsigned char c : id)
    if (!(std::isalnum(c) || c == '_' || c == '-' || c == '.'))
      return false;
  return true;
}

} // namespace

bool ParseSampleRequest(const Json &root, SampleRequest *out, std::string *error)
{
  if (!HasExactly(root, {"protocol", "mesh_artifact_path", "mesh_artifact_sha256", "circuit_currents_A",
                         "force_group_number", "stress_air_group_number", "airgap_radius_mm",
                         "airgap_angles_deg", "sliding_band_angle_deg", "compute_force_torque",
                         "include_field_solution"},
                  error))
    return false;
  const Json *protocol = root.get("protocol", K::String, error);
  const Json *path = root.get("mesh_artifact_path", K::String, error);
  const Json *sha = root.get("mesh_artifact_sha256", K::String, error);
  const Json *currents = root.get("circuit_currents_A", K::Array, error);
  const Json *force = root.get("force_group_number", K::Number, error);
  const Json *air = root.get("stress_air_group_number", K::Number, error);
  const Json *radius = root.get("airgap_radius_mm", K::Number, error);
  const Json *angles = root.get("airgap_angles_deg", K::Array, error);
  const Json *sliding = root.get("sliding_band_angle_deg", K::Number, error);
  const Json *compute = root.get("compute_force_torque", K::Bool, error);
  const Json *include = root.get("include_field_solution", K::Bool, error);
  SampleRequest r;
  int32_t selected = -2, air_group = -2;
  const bool ok = protocol && path && sha && currents && force && air && radius && angles && sliding &&
                  compute && include &&
                  (protocol->text == "gpu_femm_planar_dc_sample_v1" ||
                   protocol->text == "gpu_femm_magnetostatic_sample_v1") &&
                  !path->text.empty() && IsSha256Hex(sha->text) && AsInt32(*force, &selected) &&
                  AsInt32(*air, &air_group) && selected >= -1 && air_group >= -1 &&
                  (selected == -1) == (air_group == -1) && !(selected >= 0 && selected == air_group) &&
                  radius->number >= 0.0 && NumberArray(*currents, &r.circuit_currents_a) &&
                  NumberArray(*angles, &r.airgap_angles_deg) &&
                  (r.airgap_angles_deg.empty() || radius->number > 0.0);
  if (!ok) {
    if (error->empty())
      *error = "invalid gpu_femm_planar_dc_sample_v1 request";
    return false;
  }
  r.protocol = protocol->text;
  r.mesh_artifact_path = path->text;
  r.mesh_artifact_sha256 = sha->text;
  r.force_group_number = selected;
  r.stress_air_group_number = air_group;
  r.airgap_radius_mm = radius->number;
  r.sliding_band_angle_deg = sliding->number;
  r.compute_force_torque = compute->boolean;
  r.include_field_solution = include->boolean;
  *out = std::move(r);
  return true;
}

bool ParseSampleRequestText(const std::string &text, SampleRequest *out, std::string *error)
{
  Json root;
  return ParseJson(text, &root, error) && ParseSampleRequest(root, out, error);
}

bool ParseBatchRequestText(const std::string &text, BatchRequest *out, std::string *error)
{
  Json root;
  if (!ParseJson(text, &root, error) || !HasExactly(root, {"protocol", "max_items_per_chunk", "items"}, error))
    return false;
  const Json *protocol = root.get("protocol", K::String, error);
  const Json *chunk = root.get("max_items_per_chunk", K::Number, error);
  const Json *items = root.get("items", K::Array, error);
  BatchRequest b;
  if (!protocol || !chunk || !items || protocol->text != "gpu_femm_magnetostatic_batch_v1" ||
      !AsInt32(*chunk, &b.max_items_per_chunk) || b.max_items_per_chunk < 1 ||
      b.max_items_per_chunk > 4096 || items->items.empty() || items->items.size() > 4096) {
    if (error->empty())
      *error = "invalid gpu_femm_magnetostatic_batch_v1 request";
    return false;
  }
  b.protocol = protocol->text;
  std::set<std::string> ids;
  for (const Json &item : items->items) {
    if (!HasExactly(item, {"task_id", "request"}, error))
      return false;
    const Json *id = item.get("task_id", K::String, error);
    const Json *req = item.get("request", K::Object, error);
    BatchItem parsed;
    if (!id || !req || !TaskIdValid(id->text) || ids.count(id->text) ||
        !ParseSampleRequest(*req, &parsed.request, error)) {
      if (error->empty())
        *error = "invalid or duplicate batch task_id";
      return false;
    }
    parsed.task_id = id->text;
    ids.insert(parsed.task_id);
    b.items.push_back(std::move(parsed));
  }
  *out = std::move(b);
  return true;
}

} // namespace fgio
