// motor.h -- the production motor adapters over the conforming motor artifacts:
// --motor-single-sample, --motor-batch / --motor-batch-profile, and motor batches in the
// streaming worker.
#pragma once

#include "cli_common.h"
#include "motor_request.h"

#include <chrono>
#include <string>

namespace fgcli
{

// MotorSingleSampleAdapter (gpu_solver/src/app/sample_adapter.cpp:135-179).
int MotorSingleSample(const std::string &request_path, const std::string &response_path, const Options &opt);

// MotorBatchAdapter (gpu_solver/src/app/motor_batch.cpp:32-491): solves a parsed motor batch
// and returns the response text; `artifacts` supplies and keeps prepared artifacts.
std::string RunMotorBatch(const fgio::MotorBatchRequest &batch, const Options &opt, ArtifactCache *artifacts,
                          bool include_timing, std::chrono::steady_clock::time_point t0, bool *all_pass);

// --motor-batch / --motor-batch-profile: the exit code of the reference adapter.
int MotorBatch(const std::string &request_path, const std::string &response_path, const Options &opt,
               bool include_timing);

} // namespace fgcli
