// request.h -- sample requests and the shared-geometry batch envelope of the femm_gpu CLI.
#pragma once

#include "json.h"

#include <string>
#include <vector>

namespace fgio
{

// gpu_femm_planar_dc_sample_v1 / gpu_femm_magnetostatic_sample_v1
// (ReadPlanarDcSampleRequestJson, gpu_solver/src/io/sample_request.cpp:153-210).
struct SampleRequest {
  std::string protocol, mesh_artifact_path, mesh_artifact_sha256;
  std::vector<double> circuit_currents_a;
  int32_t force_group_number = -1, stress_air_group_number = -1;
  double airgap_radius_mm = 0.0;
  std::vector<double> airgap_angles_deg;
  double sliding_band_angle_deg = 0.0;
  bool compute_force_torque = false, include_field_solution = false;

  bool generic() const { return protocol == "gpu_femm_magnetostatic_sample_v1"; }
  bool postprocess_requested() const { return compute_force_torque || !airgap_angles_deg.empty(); }
};

bool ParseSampleRequest(const Json &root, SampleRequest *out, std::string *error);
bool ParseSampleRequestText(const std::string &text, SampleRequest *out, std::string *error);

// gpu_femm_magnetostatic_batch_v1: {protocol, max_items_per_chunk, items: [{task_id, request}]},
// the envelope rules of the reference's motor batch (gpu_solver/src/app/batch_prepare.cpp:
// 67-131): 1..4096 items and chunk width, unique task ids of [A-Za-z0-9_.-]{1,256}, every
// item of the batch protocol's sample version.
struct BatchItem {
  std::string task_id;
  SampleRequest request;
};
struct BatchRequest {
  std::string protocol;
  int32_t max_items_per_chunk = 0;
  std::vector<BatchItem> items;
};

bool ParseBatchRequestText(const std::string &text, BatchRequest *out, std::string *error);

} // namespace fgio
