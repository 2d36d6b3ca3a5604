// worker.h -- the streaming batch worker of the femm_gpu CLI (`--worker`, `--motor-worker`).
#pragma once

#include "cli_common.h"
#include "motor_request.h"
#include "request.h"

#include <chrono>
#include <functional>
#include <iosfwd>
#include <string>

namespace fgcli
{

// One transaction of the stream after admission: its envelope fields, the parsed batch
// (neutral or motor protocol) and the artifacts read for it ahead of the GPU work.
struct StreamTransaction {
  std::string session, request_path, response_path, request_sha256;
  int32_t sequence = 0;
  std::string refusal;          // empty when admitted
  bool motor = false;           // a gpu_femm_motor_batch_v* transaction
  fgio::BatchRequest neutral;   // when !motor
  fgio::MotorBatchRequest motor_batch; // when motor
  ArtifactCache staged;         // artifacts read for it that the resident set lacks, or failed checks
  double prepare_seconds = 0.0; // 0 for a refused transaction
  std::chrono::steady_clock::time_point prepare_begin, prepare_end;
};

// Solves an admitted transaction against `artifacts` (the resident plans it names) and
// returns its response text; *pass is false when any item failed.
using TransactionSolver =
    std::function<std::string(const StreamTransaction &txn, ArtifactCache *artifacts, bool *pass)>;

// Serves job envelopes from `in` (one JSON object per line) until end of input, writing
// one status line per envelope to `out`; always returns 0 (the process exit code).
int ServeStream(std::istream &in, std::ostream &out, const Options &opt, const std::string &executable,
                const TransactionSolver &solve);

} // namespace fgcli
