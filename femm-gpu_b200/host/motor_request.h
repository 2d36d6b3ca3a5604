// motor_request.h -- the production motor protocols: gpu_femm_motor_sample_v1..v4 requests and
// the gpu_femm_motor_batch_v1..v4 envelope.
#pragma once

#include "artifact.h"
#include "json.h"

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace fgio
{

// ReadMotorSampleRequestValue (gpu_solver/src/io/sample_request.cpp:212-382).
struct MotorSampleRequest {
  std::string protocol = "gpu_femm_motor_sample_v1";
  std::string mesh_artifact_path, mesh_artifact_sha256, base_motor_fem_sha256, source_fem_sha256;
  std::vector<double> circuit_currents_a;
  int32_t selected_group_number = -1, air_group_number = -1;
  double airgap_radius_mm = 0.0;
  std::vector<double> airgap_angles_deg;
  double rotor_angle_deg = 0.0, displacement_mm[2] = {0.0, 0.0};
  // v2+: gpu_femm_tangent_multi_rhs_v1 -- named circuit-current derivative directions.
  bool tangent_requested = false;
  std::vector<std::pair<std::string, std::vector<double>>> tangent_rhs;
  // v3 / v4: the sector-performance request.
  bool sector_performance = false;
  std::string model_invariance_certificate_sha256;
};

bool ParseMotorSampleRequest(const Json &root, MotorSampleRequest *out, std::string *error);
bool ParseMotorSampleRequestText(const std::string &text, MotorSampleRequest *out, std::string *error);

// RequestMatchesArtifact (sample_request.cpp:393-446) for the conforming artifacts served
// here: the request's identities, pose and circuit count against the artifact's; a v3
// request needs a v3 sector artifact with consistent harmonic metadata and the same model
// invariance certificate.  Native air-gap element sectors (v4) are not served and never
// match.
bool MotorRequestMatchesArtifact(const MotorSampleRequest &r, const Artifact &a);

// ReadMotorBatchRequestJson (gpu_solver/src/app/batch_prepare.cpp:73-129).
struct MotorBatchItem {
  std::string task_id;
  MotorSampleRequest request;
};
struct MotorBatchRequest {
  std::string protocol;
  int32_t max_items_per_chunk = 0;
  std::vector<MotorBatchItem> items;
};
bool ParseMotorBatchRequestText(const std::string &text, MotorBatchRequest *out, std::string *error);

} // namespace fgio
