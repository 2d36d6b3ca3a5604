// cli.cpp -- femm_gpu: the JSON request / response boundary of libfemmgpu.
//
//   femm_gpu [options] --solve REQUEST.json RESPONSE.json
//   femm_gpu [options] --batch BATCH.json RESPONSE.json
//   femm_gpu [options] --single-sample REQUEST.json RESPONSE.json
//   femm_gpu [options] --worker        (job envelopes on stdin, one status line per job; also --motor-worker)
//   femm_gpu [options] --motor-single-sample REQUEST.json RESPONSE.json
//   femm_gpu [options] --motor-batch[-profile] BATCH.json RESPONSE.json
//   femm_gpu --capabilities
//   femm_gpu --describe-artifact ARTIFACT.json [ROTOR_DEG]   (parsed model and plan sizes, as JSON)
//   femm_gpu --sha256 FILE                        (the file-bytes SHA-256 a request names)
//   femm_gpu --describe-femm-ans STEM CURVE_DIR   (the model --single-sample reads, as JSON)
//   options: --preconditioner jacobi|block-jacobi  --block-size 8|32  --precision fp64|mixed
//
// --solve is the reference's `--solve` (PlanarDcSingleSampleAdapter, gpu_solver/src/app/
// sample_adapter.cpp:407-489): a gpu_femm_planar_dc_sample_v1 or
// gpu_femm_magnetostatic_sample_v1 request naming a mesh artifact bound by the SHA-256 of
// its bytes; the response carries PASS / FAIL, the solve status name, flux linkage and,
// on request, the field solution; it is written to a temporary file and published by an
// atomic rename.  --batch solves a shared-geometry batch (gpu_femm_magnetostatic_batch_v1,
// the envelope of the reference's motor batch): items naming the same artifact are read
// and validated once and solved together in fg_solve_batch launches of up to
// max_items_per_chunk items; responses keep the input order.
//
// A planar-DC request with compute_force_torque or air-gap angles gets the weighted-stress
// force / torque on its force group (air = its stress-air group) and the FEMM-smoothed
// radial B on the air-gap circle (ComputeFrozenPostprocess, sample_adapter.cpp:423-439:
// mask PCG of at most 4096 iterations at 1e-12); items of a batch that share an artifact
// and the same postprocess request share one mask.
//
// --single-sample is the reference's frozen FEMM adapter (SingleSampleAdapter,
// gpu_solver/tests/native/reference_adapter.cu:63-124): a gpu_femm_single_sample_v1 request
// naming a FEMM .ans nonlinear PM / coil solution, solved from scratch (relative tolerance
// 1e-8, at most 128 Newton iterations, the other NonlinearOptions defaults), then
// postprocessed on material label 1 with label 3 as air.
//
// Exit codes: 0 every response PASS, 1 a FAIL response or an I/O failure, 2 usage error.
#include "artifact.h"
#include "cli_common.h"
#include "motor.h"
#include "femm_ans.h"
#include "femm_gpu.h"
#include "json.h"
#include "request.h"
#include "worker.h"

#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <vector>

namespace
{

using namespace fgcli;
using fgio::Artifact;
using fgio::SampleRequest;

// WritePlanarDcSampleResponse's layout (gpu_solver/src/app/sample_adapter.cpp:236-355).
std::string SampleResponse(int status, int solve_status, bool post_requested, int post_status,
                           const SampleRequest *req, const Solved *sol, const std::string &diagnostic,
                           const Artifact *art, const std::string &indent = "", const Post *post = nullptr)
{
  std::ostringstream o;
  o << std::setprecision(17);
  const bool solved = solve_status == 0 && req && sol;
  const bool postprocessed = solved && post_requested && post_status == 0 && post;
  const std::string protocol = req ? req->protocol : "gpu_femm_planar_dc_sample_v1";
  const bool generic = protocol == "gpu_femm_magnetostatic_sample_v1";
  const bool axi = art && art->problem_type == FG_AXISYMMETRIC;
  const std::string message = status == 0 ? "" : (diagnostic.empty() ? StatusName(status) : diagnostic);
  const std::string in = indent + "  ";
  o << "{\n" << in << "\"protocol\": \"" << protocol << "\",\n"
    << in << "\"mesh_artifact_sha256\": \"" << (req ? req->mesh_artifact_sha256 : "") << "\",\n";
  if (generic)
    o << in << "\"problem_type\": \"" << (axi ? "axisymmetric" : "planar") << "\",\n"
      << in << "\"field_components\": [\"" << (axi ? "Br" : "Bx") << "\", \"" << (axi ? "Bz" : "By") << "\"],\n"
      << in << "\"node_potential_quantity\": \"" << (axi ? "poloidal_flux_function" : "magnetic_vector_potential") << "\",\n"
      << in << "\"node_potential_unit\": \"" << (axi ? "Wb" : "Wb/m") << "\",\n";
  o << in << "\"status\": \"" << (status == 0 ? "PASS" : "FAIL") << "\",\n"
    << in << "\"solve_status\": \"" << StatusName(solve_status) << "\",\n"
    << in << "\"postprocess_status\": \""
    << (!post_requested ? "NOT_REQUESTED" : (solve_status == 0 ? StatusName(post_status) : "NOT_RUN")) << "\",\n"
    << in << "\"error_identifier\": \"" << (status == 0 ? "" : "GPU_FEMM_" + StatusName(status)) << "\",\n"
    << in << "\"error_message\": \"" << fgio::Escape(message) << "\",\n";
  if (postprocessed && req->compute_force_torque)
    o << in << "\"Fx_N\": " << post->fx << ",\n" << in << "\"Fy_N\": " << post->fy << ",\n"
      << in << "\"torque_Nm\": " << post->torque << ",\n";
  else
    o << in << "\"Fx_N\": null,\n" << in << "\"Fy_N\": null,\n" << in << "\"torque_Nm\": null,\n";
  o << in << "\"actual_circuit_currents_A\": [";
  if (solved)
    List(o, sol->currents);
  o << "],\n" << in << "\"circuit_flux_linkage_Wb\": [";
  if (solved)
    List(o, sol->flux);
  o << "],\n" << in << "\"airgap_sample_angles_deg\": [";
  if (postprocessed)
    List(o, req->airgap_angles_deg);
  o << "],\n" << in << "\"airgap_radial_flux_density_T\": [";
  if (postprocessed)
    List(o, post->radial);
  o << "],\n" << in << "\"mesh_node_count\": " << (solved ? sol->a.size() : 0) << ",\n"
    << in << "\"mesh_element_count\": " << (solved ? sol->b1.size() : 0) << ",\n";
  const bool field = solved && req->include_field_solution;
  o << in << "\"field_solution_included\": " << (field ? "true" : "false") << ",\n"
    << in << "\"" << (generic ? "node_potential" : "node_A_Wb_per_m") << "\": [";
  if (field)
    for (size_t i = 0; i < sol->a.size(); ++i) {
      double v = sol->a[i];
      if (generic && axi && art && 2 * i < art->xy.size())
        v *= kTwoPi * art->xy[2 * i];
      o << (i ? ", " : "") << v;
    }
  o << "],\n" << in << "\"" << (generic ? "element_B_component_1_T" : "element_Bx_T") << "\": [";
  if (field)
    List(o, sol->b1);
  o << "],\n" << in << "\"" << (generic ? "element_B_component_2_T" : "element_By_T") << "\": [";
  if (field)
    List(o, sol->b2);
  o << "],\n" << in << "\"convergence\": {\"iterations\": " << (sol ? sol->iterations : 0) << ", \"residual_l2\": ";
  if (sol && std::isfinite(sol->residual))
    o << sol->residual;
  else
    o << "null";
  o << "}\n" << indent << "}";
  return o.str();
}

// PlanarDcRequestMatchesArtifact (sample_adapter.cpp:181-234): the generic protocol on
// generic artifacts (field solve only), the planar-DC protocol on the others; a sliding-band
// artifact takes any sliding_band_angle_deg and needs the probe circle inside every band.
bool RequestMatchesArtifact(const SampleRequest &r, const Artifact &a)
{
  const bool generic_artifact = a.schema_version == "gpu_femm_magnetostatic_mesh_v1";
  if (r.generic() != generic_artifact || r.circuit_currents_a.size() != a.circuit_currents.size())
    return false;
  auto has_group = [&](int32_t g) {
    for (int32_t x : a.group_numbers)
      if (x == g)
        return true;
    return false;
  };
  const bool groups = r.force_group_number >= 0;
  if (groups && (!has_group(r.force_group_number) || !has_group(r.stress_air_group_number)))
    return false;
  const bool post = r.postprocess_requested();
  if (r.generic())
    return !post && r.force_group_number == -1 && r.stress_air_group_number == -1 &&
           r.airgap_radius_mm == 0.0 && r.airgap_angles_deg.empty() && r.sliding_band_angle_deg == 0.0;
  if (!a.sliding_band)
    return r.sliding_band_angle_deg == 0.0 && (!post || groups);
  if (!r.airgap_angles_deg.empty()) {
    if (a.bands.empty())
      return false;
    for (const fgio::AirGapBand &b : a.bands) {
      const double ri = 1000.0 * b.ri_m, ro = 1000.0 * b.ro_m, tol = 1e-9 * std::max(1.0, std::abs(ro));
      if (r.airgap_radius_mm < ri - tol || r.airgap_radius_mm > ro + tol)
        return false;
    }
  }
  return true;
}

// The postprocess of one planar-DC sample: the band's for a sliding-band artifact, else the
// weighted-stress one (sample_adapter.cpp:426-439).
int PostSample(Prepared &p, const SampleRequest &r, const Solved &sol, Post *out)
{
  if (p.artifact.sliding_band)
    return AirGapPost(p.plan, sol, r.airgap_angles_deg, out);
  fg_postprocess *pp = nullptr;
  const int rc = p.post.Get(p.plan, r.force_group_number, r.stress_air_group_number, r.airgap_radius_mm,
                            r.airgap_angles_deg, &pp);
  return rc != 0 ? rc : RunPost(pp, sol, out);
}

// Solves k samples on a prepared plan; statuses[i] = per-item status.
int SolveItems(Prepared &p, const std::vector<const SampleRequest *> &reqs, std::vector<Solved> *out,
               std::vector<int> *statuses, int *launches)
{
  std::vector<const std::vector<double> *> currents;
  for (const SampleRequest *r : reqs)
    currents.push_back(&r->circuit_currents_a);
  return SolveCurrents(p, currents, out, statuses, launches);
}

int Solve(const std::string &request_path, const std::string &response_path, const Options &opt)
{
  if (SameFile(request_path, response_path)) {
    std::cerr << "FAIL magnetostatic solve: response must not overwrite request\n";
    return 1;
  }
  std::string text, error;
  SampleRequest req;
  const bool read = ReadFile(request_path, &text);
  const bool parsed = read && fgio::ParseSampleRequestText(text, &req, &error);
  if (parsed && SameFile(req.mesh_artifact_path, response_path)) {
    std::cerr << "FAIL magnetostatic solve: response must not overwrite mesh artifact\n";
    return 1;
  }
  if (!parsed) {
    if (!read)
      error = "cannot read request";
    const std::string body =
        SampleResponse(FG_INVALID_ARGUMENT, FG_INVALID_ARGUMENT, false, 0, nullptr, nullptr, error, nullptr);
    if (!PublishAtomically(response_path, body + "\n")) {
      std::cerr << "FAIL magnetostatic solve: could not atomically publish response\n";
      return 1;
    }
    std::cerr << "FAIL planar-DC request: " << error << '\n';
    return 1;
  }
  Prepared base;
  Prepare(req.mesh_artifact_path, req.mesh_artifact_sha256, opt, &base);
  int status = base.status;
  std::string diagnostic = base.error;
  if (status == 0 && !RequestMatchesArtifact(req, base.artifact)) {
    status = FG_INVALID_ARGUMENT;
    diagnostic = "artifact physics, circuit count, group, or sliding-band request mismatch";
  }
  // ApplySlidingBandAngle (sample_adapter.cpp:404-408): a sliding-band artifact is solved at
  // the request's band angle.
  Prepared &p = status == 0 ? *PoseOf(base, req.sliding_band_angle_deg) : base;
  if (status == 0 && p.status != 0) {
    status = p.status;
    diagnostic = p.error;
  }
  std::vector<Solved> sols;
  std::vector<int> st;
  int launches = 0;
  bool attempted = false;
  if (status == 0)
    status = EnsurePlan(&p, opt);
  if (status == 0) {
    attempted = true;
    const int rc = SolveItems(p, {&req}, &sols, &st, &launches);
    status = rc != 0 ? rc : st[0];
  }
  const int solve_status = status;
  const bool post = req.postprocess_requested();
  int post_status = 0;
  Post result;
  if (solve_status == 0 && post) {
    post_status = PostSample(p, req, sols[0], &result);
    status = post_status;
  }
  const std::string body = SampleResponse(status, solve_status, post, post_status, &req,
                                          attempted ? &sols[0] : nullptr, diagnostic, &p.artifact, "",
                                          post_status == 0 ? &result : nullptr);
  if (!PublishAtomically(response_path, body + "\n")) {
    std::cerr << "FAIL magnetostatic solve: could not atomically publish response\n";
    return 1;
  }
  if (status != 0) {
    std::cerr << "FAIL magnetostatic solve: " << (diagnostic.empty() ? StatusName(status) : diagnostic) << '\n';
    return 1;
  }
  return 0;
}

// Solves the ready items of one operator (an artifact, or one band angle of a sliding-band
// artifact) in chunks of max_items_per_chunk and writes their response bodies.
// given / given_status: the pose's samples already solved (with other poses, in one
// multi-plan launch); then only the postprocess and the responses remain.
void SolvePose(const fgio::BatchRequest &batch, const Options &opt, Prepared &p, const std::vector<size_t> &ready,
               std::vector<std::string> *bodies, std::vector<int> *final_status, int *chunks, int *launches,
               double *solve_s, const std::vector<Solved> *given = nullptr,
               const std::vector<int> *given_status = nullptr)
{
  const int plan_status = p.status != 0 ? p.status : EnsurePlan(&p, opt);
  if (plan_status != 0) {
    for (size_t i : ready) {
      const SampleRequest &r = batch.items[i].request;
      (*bodies)[i] = SampleResponse(plan_status, plan_status, r.postprocess_requested(), 0, &r, nullptr, p.error,
                                    nullptr, "    ");
      (*final_status)[i] = plan_status;
    }
    return;
  }
  const auto s0 = std::chrono::steady_clock::now();
  for (size_t first = 0; first < ready.size(); first += batch.max_items_per_chunk) {
    const size_t n = std::min<size_t>(batch.max_items_per_chunk, ready.size() - first);
    std::vector<const SampleRequest *> reqs;
    for (size_t j = 0; j < n; ++j)
      reqs.push_back(&batch.items[ready[first + j]].request);
    std::vector<Solved> sols;
    std::vector<int> st;
    if (given) {
      sols.assign(given->begin() + first, given->begin() + first + n);
      st.assign(given_status->begin() + first, given_status->begin() + first + n);
    } else {
      SolveItems(p, reqs, &sols, &st, launches);
    }
    ++*chunks;
    for (size_t j = 0; j < n; ++j) {
      const size_t i = ready[first + j];
      const SampleRequest &r = *reqs[j];
      int status = st[j];
      const int solve_status = status;
      int post_status = 0;
      Post result;
      if (solve_status == 0 && r.postprocess_requested()) {
        post_status = PostSample(p, r, sols[j], &result);
        status = post_status;
      }
      (*bodies)[i] = SampleResponse(status, solve_status, r.postprocess_requested(), post_status, &r,
                                    sols.empty() ? nullptr : &sols[j], "", &p.artifact, "    ",
                                    post_status == 0 ? &result : nullptr);
      (*final_status)[i] = status;
    }
  }
  *solve_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
}

// Solves a parsed batch and returns the response text.  Items naming the same artifact are
// solved together; `artifacts` supplies prepared artifacts (and keeps the ones prepared
// here), so a caller that keeps it keeps plans and postprocess masks across batches.
std::string RunBatch(const fgio::BatchRequest &batch, const Options &opt, ArtifactCache *artifacts,
                     std::chrono::steady_clock::time_point t0, bool *all_pass)
{
  const size_t k = batch.items.size();
  std::vector<std::string> bodies(k);
  std::vector<int> final_status(k, FG_INTERNAL_ERROR);
  // Items grouped by artifact (path + SHA): each artifact read, verified and planned once.
  std::map<ArtifactKey, std::vector<size_t>> groups;
  for (size_t i = 0; i < k; ++i)
    groups[{batch.items[i].request.mesh_artifact_path, batch.items[i].request.mesh_artifact_sha256}].push_back(i);
  int chunks = 0, launches = 0, cache_hits = 0;
  double artifact_s = 0.0, solve_s = 0.0;
  for (auto &g : groups) {
    cache_hits += static_cast<int>(g.second.size()) - 1;
    const auto a0 = std::chrono::steady_clock::now();
    std::shared_ptr<Prepared> &slot = (*artifacts)[g.first];
    if (!slot) {
      slot = std::make_shared<Prepared>();
      Prepare(g.first.first, g.first.second, opt, slot.get());
    }
    Prepared &p = *slot;
    artifact_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - a0).count();
    std::vector<size_t> ready;
    for (size_t i : g.second) {
      const SampleRequest &r = batch.items[i].request;
      int status = p.status;
      std::string diag = p.error;
      if (status == 0 && !RequestMatchesArtifact(r, p.artifact)) {
        status = FG_INVALID_ARGUMENT;
        diag = "artifact physics, circuit count, group, or sliding-band request mismatch";
      }
      if (status == 0) {
        ready.push_back(i);
        continue;
      }
      bodies[i] = SampleResponse(status, status, r.postprocess_requested(), 0, &r, nullptr, diag, nullptr, "    ");
      final_status[i] = status;
    }
    // A sliding-band artifact has one operator per band angle: its items are solved per pose.
    TrimPoses(p, kResidentPoses);
    std::map<double, std::vector<size_t>> poses;
    for (size_t i : ready)
      poses[p.artifact.sliding_band ? batch.items[i].request.sliding_band_angle_deg : 0.0].push_back(i);
    // Several poses of a sliding-band artifact: their samples in one multi-plan launch per
    // Newton step when SolveOperatorsTogether applies, else pose by pose.
    std::vector<Operator> ops;
    for (auto &pose : poses) {
      Operator op{PoseOf(p, pose.first), {}};
      for (size_t i : pose.second)
        op.currents.push_back(&batch.items[i].request.circuit_currents_a);
      ops.push_back(std::move(op));
    }
    std::vector<std::vector<Solved>> together;
    std::vector<std::vector<int>> together_status;
    int64_t unused_pcg = 0;
    const auto m0 = std::chrono::steady_clock::now();
    const bool joint = batch.max_items_per_chunk >= static_cast<int32_t>(ready.size()) &&
                       SolveOperatorsTogether(ops, opt, &together, &together_status, &launches, &unused_pcg);
    if (joint)
      solve_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - m0).count();
    size_t o = 0;
    for (auto &pose : poses) {
      SolvePose(batch, opt, *ops[o].p, pose.second, &bodies, &final_status, &chunks, &launches, &solve_s,
                joint ? &together[o] : nullptr, joint ? &together_status[o] : nullptr);
      ++o;
    }
  }
  bool &pass = *all_pass;
  pass = true;
  for (int s : final_status)
    pass = pass && s == 0;
  std::ostringstream o;
  o << std::setprecision(17) << "{\n  \"protocol\": \"" << batch.protocol << "\",\n"
    << "  \"status\": \"" << (pass ? "PASS" : "FAIL") << "\",\n"
    << "  \"solve_status\": \"" << (pass ? "PASS" : "PARTIAL_FAILURE") << "\",\n"
    << "  \"error_identifier\": \"" << (pass ? "" : "GPU_FEMM_BATCH_PARTIAL_FAILURE") << "\",\n"
    << "  \"error_message\": \"" << (pass ? "" : "one or more batch items failed") << "\",\n"
    << "  \"cache\": {\"mesh_cache_hits\": " << cache_hits << ", \"chunk_count\": " << chunks
    << ", \"requested_chunk_size\": " << batch.max_items_per_chunk
    << ", \"effective_chunk_size\": " << batch.max_items_per_chunk
    << ", \"batched_pcg_launches\": " << launches << "},\n"
    << "  \"timing\": {\"schema_version\": \"gpu_femm_magnetostatic_batch_timing_v1\""
    << ", \"artifact_read_validate_plan_seconds\": " << artifact_s << ", \"solve_seconds\": " << solve_s
    << ", \"total_seconds\": " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
    << "},\n  \"items\": [\n";
  for (size_t i = 0; i < k; ++i)
    o << "    {\"task_id\": \"" << batch.items[i].task_id << "\", \"response\": " << bodies[i]
      << (i + 1 < k ? "},\n" : "}\n");
  o << "  ]\n}\n";
  return o.str();
}

int Batch(const std::string &request_path, const std::string &response_path, const Options &opt)
{
  if (SameFile(request_path, response_path)) {
    std::cerr << "FAIL magnetostatic batch: response must not overwrite request\n";
    return 1;
  }
  const auto t0 = std::chrono::steady_clock::now();
  std::string text, error;
  fgio::BatchRequest batch;
  if (!ReadFile(request_path, &text) || !fgio::ParseBatchRequestText(text, &batch, &error)) {
    std::ostringstream o;
    o << "{\n  \"protocol\": \"gpu_femm_magnetostatic_batch_v1\",\n  \"status\": \"FAIL\",\n"
      << "  \"solve_status\": \"" << StatusName(FG_INVALID_ARGUMENT) << "\",\n"
      << "  \"error_identifier\": \"GPU_FEMM_" << StatusName(FG_INVALID_ARGUMENT) << "\",\n"
      << "  \"error_message\": \"" << fgio::Escape(error.empty() ? "cannot read request" : error)
      << "\",\n  \"items\": []\n}\n";
    PublishAtomically(response_path, o.str());
    std::cerr << "FAIL magnetostatic batch request: " << error << '\n';
    return 1;
  }
  ArtifactCache artifacts;
  bool pass = false;
  const std::string text_out = RunBatch(batch, opt, &artifacts, t0, &pass);
  if (!PublishAtomically(response_path, text_out)) {
    std::cerr << "FAIL magnetostatic batch: could not atomically publish response\n";
    return 1;
  }
  if (!pass)
    std::cerr << "FAIL magnetostatic batch: one or more batch items failed\n";
  return pass ? 0 : 1;
}

// ---- --worker: the streaming batch worker (host/worker.cpp).  Each admitted transaction
// is solved by the one-shot adapters' code against the worker's resident artifacts; motor
// transactions carry the reference worker's timing block.
int Worker(const Options &opt, const std::string &executable)
{
  return ServeStream(std::cin, std::cout, opt, executable,
                     [&opt](const StreamTransaction &txn, ArtifactCache *artifacts, bool *pass) {
                       return txn.motor ? RunMotorBatch(txn.motor_batch, opt, artifacts, true, txn.prepare_begin, pass)
                                        : RunBatch(txn.neutral, opt, artifacts, txn.prepare_begin, pass);
                     });
}

// WriteSingleSampleResponse (gpu_solver/tests/native/reference_adapter.cu:16-61).
std::string SingleSampleResponse(int status, const fgio::SingleSampleRequest *req, const Solved *sol,
                                 const Post *post)
{
  std::ostringstream o;
  o << std::setprecision(17) << "{\n  \"protocol\": \"gpu_femm_single_sample_v1\",\n"
    << "  \"source_motor_fem_sha256\": \"" << (req ? req->source_motor_fem_sha256 : "") << "\",\n"
    << "  \"status\": \"" << (status == 0 ? "PASS" : "FAIL") << "\",\n"
    << "  \"solve_status\": \"" << (status == 0 ? "PASS" : "FAIL") << "\",\n"
    << "  \"error_identifier\": \"" << (status == 0 ? "" : "GPU_FEMM_" + StatusName(status)) << "\",\n"
    << "  \"error_message\": \"" << (status == 0 ? "" : StatusName(status)) << "\",\n";
  if (status == 0 && req && sol && post) {
    o << "  \"Fx_N\": " << post->fx << ",\n  \"Fy_N\": " << post->fy << ",\n  \"torque_Nm\": " << post->torque
      << ",\n  \"actual_circuit_currents_A\": [" << req->current_a << "],\n  \"circuit_flux_linkage_Wb\": ["
      << sol->flux[0] << "],\n  \"airgap_sample_angles_deg\": [";
    List(o, req->airgap_angles_deg);
    o << "],\n  \"airgap_radial_flux_density_T\": [";
    List(o, post->radial);
    o << "],\n  \"mesh_element_count\": " << sol->b1.size() << ",\n  \"convergence\": {\"iterations\": "
      << sol->iterations << ", \"residual_l2\": " << sol->residual << "}\n";
  } else {
    o << "  \"Fx_N\": null,\n  \"Fy_N\": null,\n  \"torque_Nm\": null,\n"
      << "  \"actual_circuit_currents_A\": [],\n  \"circuit_flux_linkage_Wb\": [],\n"
      << "  \"airgap_sample_angles_deg\": [],\n  \"airgap_radial_flux_density_T\": [],\n"
      << "  \"mesh_element_count\": 0,\n  \"convergence\": {\"iterations\": 0, \"residual_l2\": null}\n";
  }
  o << "}\n";
  return o.str();
}

int SingleSample(const std::string &request_path, const std::string &response_path, const Options &opt)
{
  std::string text, error;
  // A strict-JSON gpu_femm_motor_sample_v1 request goes to the motor adapter
  // (SingleSampleAdapter, reference_adapter.cu:63-78).
  {
    fgio::Json root;
    std::string ignored;
    if (ReadFile(request_path, &text) && fgio::ParseJson(text, &root, &ignored) && root.is(fgio::Json::Kind::Object)) {
      auto it = root.members.find("protocol");
      if (it != root.members.end() && it->second.is(fgio::Json::Kind::String) &&
          it->second.text == "gpu_femm_motor_sample_v1")
        return MotorSingleSample(request_path, response_path, opt);
    }
    text.clear();
  }
  fgio::SingleSampleRequest req;
  if (!ReadFile(request_path, &text) || !fgio::ParseSingleSampleRequestText(text, &req, &error)) {
    if (!PublishAtomically(response_path, SingleSampleResponse(FG_INVALID_ARGUMENT, nullptr, nullptr, nullptr))) {
      std::cerr << "FAIL single-sample response: cannot write " << response_path << '\n';
      return 1;
    }
    std::cerr << "FAIL single-sample request: " << (error.empty() ? "cannot read request" : error) << '\n';
    return 1;
  }
  Prepared p;
  std::vector<double> femm_a;
  bool loaded = fgio::ReadFemmNonlinear(req.stem, req.curve_directory, &p.artifact, &femm_a, &error);
  if (loaded) {
    // ValidateNonlinearModel belongs to the fixture reader: a host-only plan checks it.
    fg_model m = p.artifact.Model();
    fg_plan_options host = opt.plan;
    host.flags |= FG_PLAN_HOST_ONLY;
    fg_plan *check = nullptr;
    loaded = fg_plan_create(&m, &host, &check) == 0;
    if (check)
      fg_plan_destroy(check);
    if (!loaded)
      error = "nonlinear frozen mesh validation failed";
  }
  if (!loaded) {
    if (!PublishAtomically(response_path, SingleSampleResponse(FG_INPUT_IO, &req, nullptr, nullptr))) {
      std::cerr << "FAIL single-sample response: cannot write " << response_path << '\n';
      return 1;
    }
    std::cerr << "FAIL single-sample reference: " << error << '\n';
    return 1;
  }
  int status = EnsurePlan(&p, opt);
  Solved sol;
  if (status == 0) {
    const fg_model m = p.artifact.Model();
    const size_t N = m.node_count, E = m.triangle_count;
    sol.currents = {req.current_a};
    sol.flux.assign(1, 0.0);
    sol.a.assign(N, 0.0);
    sol.b1.assign(E, 0.0);
    sol.b2.assign(E, 0.0);
    // NonlinearOptions defaults with relative tolerance 1e-8 and 128 Newton iterations.
    const fg_solve_options o{1e-8, 128, 128, 1e-13, 0, 0};
    fg_item_info info{};
    status = fg_solve_batch(p.plan, 1, sol.currents.data(), nullptr, nullptr, &o, sol.a.data(), sol.b1.data(),
                            sol.b2.data(), sol.flux.data(), &info);
    if (status == 0)
      status = info.status;
    sol.iterations = info.iterations;
    sol.residual = info.residual_l2;
  }
  Post post;
  if (status == 0) {
    std::vector<double> angles;
    for (double deg : req.airgap_angles_deg)
      angles.push_back(deg * kPi / 180.0);
    fg_postprocess_options o;
    fg_postprocess_default_options(&o);
    o.selected_material_label = req.selected_material_label;
    o.airgap_radius_m = req.airgap_radius_mm * 1e-3;
    o.airgap_angle_count = static_cast<int32_t>(angles.size());
    o.airgap_angles_rad = angles.data();
    fg_postprocess *pp = nullptr;
    status = fg_postprocess_create(p.plan, &o, nullptr, &pp);
    if (status == 0) {
      status = RunPost(pp, sol, &post);
      fg_postprocess_destroy(pp);
    }
  }
  if (!PublishAtomically(response_path, SingleSampleResponse(status, &req, status == 0 ? &sol : nullptr,
                                                             status == 0 ? &post : nullptr))) {
    std::cerr << "FAIL single-sample response: cannot write " << response_path << '\n';
    return 1;
  }
  if (status != 0) {
    std::cerr << "FAIL single-sample: " << StatusName(status) << '\n';
    return 1;
  }
  return 0;
}

// The parsed model as JSON (17 significant digits, exact round trip) with its host-only
// plan's sizes -- for checking the readers against the reference's.
int DescribeModel(Artifact &a, const std::string &sha256)
{
  fg_model m = a.Model();
  fg_plan_options po{FG_PRECOND_JACOBI, 8, FG_PRECISION_FP64, FG_PLAN_HOST_ONLY};
  fg_plan *plan = nullptr;
  const int rc = fg_plan_create(&m, &po, &plan);
  fg_plan_sizes sz{};
  if (rc == 0)
    fg_plan_sizes_get(plan, &sz);
  std::ostringstream o;
  o << std::setprecision(17) << "{\"status\": \"PASS\", \"plan_status\": \"" << StatusName(rc)
    << "\", \"schema_version\": \"" << a.schema_version << "\", \"sha256\": \"" << sha256
    << "\", \"canonical_identity_sha256\": \"" << a.canonical_identity_sha256
    << "\", \"problem_type\": " << a.problem_type << ", \"depth_m\": " << a.depth_m << ", \"xy\": [";
  List(o, a.xy);
  o << "], \"tri\": [";
  List(o, a.tri);
  o << "], \"tri_mat\": [";
  List(o, a.tri_mat);
  o << "], \"materials\": [";
  for (size_t i = 0; i < a.materials.size(); ++i) {
    const fg_material &t = a.materials[i];
    o << (i ? ", " : "") << "[" << t.reluctivity_zero_m_per_h << ", " << t.alpha_per_t2 << ", "
      << t.source_j_per_a << ", " << t.h_c_a_per_m << ", " << t.magnetization_deg << ", "
      << t.bh_curve_index << ", " << t.circuit_index << ", " << t.group_number << "]";
  }
  o << "], \"curves\": [";
  for (size_t c = 0; c < a.curve_b.size(); ++c) {
    o << (c ? ", " : "") << "[[";
    List(o, a.curve_b[c]);
    o << "], [";
    List(o, a.curve_h[c]);
    o << "]]";
  }
  o << "], \"dirichlet_nodes\": [";
  List(o, a.dir_nodes);
  o << "], \"constraint_nodes\": [";
  List(o, a.con_nodes);
  o << "], \"constraint_signs\": [";
  for (size_t i = 0; i < a.con_signs.size(); ++i)
    o << (i ? ", " : "") << static_cast<int>(a.con_signs[i]);
  o << "], \"circuit_currents_A\": [";
  List(o, a.circuit_currents);
  o << "], \"air_gap_elements\": [";
  for (size_t b = 0; b < a.bands.size(); ++b) {
    const fgio::AirGapBand &g = a.bands[b];
    o << (b ? ", " : "") << "{\"antiperiodic\": " << (g.antiperiodic ? 1 : 0) << ", \"center_m\": ["
      << g.center_m[0] << ", " << g.center_m[1] << "], \"ri_m\": " << g.ri_m << ", \"ro_m\": " << g.ro_m
      << ", \"arc_length_deg\": " << g.arc_deg << ", \"inner_shift\": " << g.inner_shift
      << ", \"outer_shift\": " << g.outer_shift << ", \"nodes\": [";
    List(o, g.nodes);
    o << "], \"weights\": [";
    List(o, g.weights);
    o << "]}";
  }
  o << "], \"rows\": " << sz.rows << ", \"nnz\": " << sz.nnz << "}\n";
  if (plan)
    fg_plan_destroy(plan);
  std::cout << o.str();
  return rc == 0 ? 0 : 1;
}

// --describe-artifact ARTIFACT.json [ROTOR_ANGLE_DEG]: a sliding-band artifact is described
// posed at the angle (its bands slid as a motor request at that angle solves them).
int DescribeArtifact(const std::string &path, const char *rotor_angle_deg = nullptr)
{
  std::string bytes, error;
  Artifact a;
  if (!ReadFile(path, &bytes)) {
    std::cerr << "FAIL describe: cannot open mesh artifact\n";
    return 1;
  }
  if (!fgio::ParseArtifact(bytes, &a, &error)) {
    std::cout << "{\"status\": \"FAIL\", \"error\": \"" << fgio::Escape(error) << "\"}\n";
    return 1;
  }
  if (rotor_angle_deg && !a.SlideBands(std::strtod(rotor_angle_deg, nullptr))) {
    std::cout << "{\"status\": \"FAIL\", \"error\": \"could not apply the requested sliding-band angle\"}\n";
    return 1;
  }
  return DescribeModel(a, fgio::Sha256Hex(bytes));
}

// --describe-femm-ans STEM CURVE_DIRECTORY: the model --single-sample solves.
int DescribeFemmAns(const std::string &stem, const std::string &curves)
{
  std::string error;
  Artifact a;
  std::vector<double> femm_a;
  if (!fgio::ReadFemmNonlinear(stem, curves, &a, &femm_a, &error)) {
    std::cout << "{\"status\": \"FAIL\", \"error\": \"" << fgio::Escape(error) << "\"}\n";
    return 1;
  }
  return DescribeModel(a, "");
}

int Usage()
{
  std::cerr << "usage: femm_gpu [--preconditioner jacobi|block-jacobi] [--block-size 8|32] "
               "[--precision fp64|mixed] (--solve request.json response.json | "
               "--batch batch.json response.json | --single-sample request.json response.json | --worker | "
               "--motor-single-sample request.json response.json | --motor-batch[-profile] batch.json response.json | "
               "--capabilities | --describe-artifact artifact.json)\n";
  return 2;
}

} // namespace

int main(int argc, char **argv)
{
  Options opt;
  int next = 1;
  bool have_pre = false, have_prec = false, have_bs = false;
  while (next + 1 < argc && (std::strcmp(argv[next], "--preconditioner") == 0 ||
                             std::strcmp(argv[next], "--block-size") == 0 ||
                             std::strcmp(argv[next], "--precision") == 0)) {
    const std::string flag = argv[next], value = argv[next + 1];
    if (flag == "--preconditioner") {
      if (have_pre || (value != "jacobi" && value != "block-jacobi")) {
        std::cerr << "--preconditioner requires jacobi or block-jacobi\n";
        return 2;
      }
      opt.plan.preconditioner = value == "block-jacobi" ? FG_PRECOND_BLOCK_JACOBI : FG_PRECOND_JACOBI;
      have_pre = true;
    } else if (flag == "--block-size") {
      if (have_bs || (value != "8" && value != "32")) {
        std::cerr << "--block-size requires 8 or 32\n";
        return 2;
      }
      opt.plan.block_size = value == "32" ? 32 : 8;
      have_bs = true;
    } else {
      if (have_prec || (value != "fp64" && value != "mixed")) {
        std::cerr << "--precision requires fp64 or mixed\n";
        return 2;
      }
      opt.plan.precision = value == "mixed" ? FG_PRECISION_MIXED : FG_PRECISION_FP64;
      have_prec = true;
    }
    next += 2;
  }
  const int rest = argc - next;
  if (rest == 1 && std::strcmp(argv[next], "--capabilities") == 0) {
    std::cout << "{\n  \"protocols\": [\"gpu_femm_planar_dc_sample_v1\", \"gpu_femm_magnetostatic_sample_v1\", "
                 "\"gpu_femm_magnetostatic_batch_v1\", \"gpu_femm_single_sample_v1\", \"gpu_femm_motor_sample_v1\", "
                 "\"gpu_femm_motor_sample_v2\", \"gpu_femm_motor_sample_v3\", \"gpu_femm_motor_sample_v4\", "
                 "\"gpu_femm_motor_batch_v1\", \"gpu_femm_motor_batch_v2\", \"gpu_femm_motor_batch_v3\", "
                 "\"gpu_femm_motor_batch_v4\"],\n"
              << "  \"mesh_artifacts\": [\"gpu_femm_planar_dc_mesh_v1\", \"gpu_femm_magnetostatic_mesh_v1\", "
                 "\"gpu_femm_mesh_v1\", \"gpu_femm_mesh_v2\", \"gpu_femm_mesh_v3\", \"gpu_femm_mesh_v4\"],\n"
              << "  \"native_sliding_band\": true,\n"
              << "  \"motor_sector_native_age_cyclic_v1\": true,\n"
              << "  \"preconditioners\": [\"jacobi\", \"block-jacobi\"],\n"
              << "  \"precisions\": [\"fp64\", \"mixed\"],\n"
              << "  \"abi_version\": " << fg_abi_version() << "\n}\n";
    return 0;
  }
  if (rest == 2 && std::strcmp(argv[next], "--sha256") == 0) {
    std::string bytes;
    if (!ReadFile(argv[next + 1], &bytes)) {
      std::cerr << "FAIL sha256: cannot read " << argv[next + 1] << '\n';
      return 1;
    }
    std::cout << fgio::Sha256Hex(bytes) << '\n';
    return 0;
  }
  if (rest == 2 && std::strcmp(argv[next], "--describe-artifact") == 0)
    return DescribeArtifact(argv[next + 1]);
  if (rest == 3 && std::strcmp(argv[next], "--describe-artifact") == 0)
    return DescribeArtifact(argv[next + 1], argv[next + 2]);
  if (rest == 3 && std::strcmp(argv[next], "--describe-femm-ans") == 0)
    return DescribeFemmAns(argv[next + 1], argv[next + 2]);
  if (rest == 3 && std::strcmp(argv[next], "--solve") == 0)
    return Solve(argv[next + 1], argv[next + 2], opt);
  if (rest == 3 && std::strcmp(argv[next], "--batch") == 0)
    return Batch(argv[next + 1], argv[next + 2], opt);
  if (rest == 1 && (std::strcmp(argv[next], "--worker") == 0 || std::strcmp(argv[next], "--motor-worker") == 0))
    return Worker(opt, argv[0]);
  if (rest == 3 && std::strcmp(argv[next], "--motor-single-sample") == 0)
    return MotorSingleSample(argv[next + 1], argv[next + 2], opt);
  if (rest == 3 && std::strcmp(argv[next], "--motor-batch") == 0)
    return MotorBatch(argv[next + 1], argv[next + 2], opt, false);
  if (rest == 3 && std::strcmp(argv[next], "--motor-batch-profile") == 0)
    return MotorBatch(argv[next + 1], argv[next + 2], opt, true);
  if (rest == 3 && std::strcmp(argv[next], "--single-sample") == 0)
    return SingleSample(argv[next + 1], argv[next + 2], opt);
  return Usage();
}
