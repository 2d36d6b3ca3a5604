// motor.cpp -- production motor adapters (see motor.h).
//
// Items of a motor batch are checked against their artifact (SHA-256 of the file bytes,
// base and source identities, the mesh's pose, circuit count), grouped by artifact within
// chunks of up to 32 items, solved in one fg_solve_batch per group with the production
// options, postprocessed on their selected / air groups (weighted-stress force and torque,
// smoothed air-gap B; the mask solved once per artifact and request options), and -- for
// gpu_femm_motor_sample_v2 items with tangent_multi_rhs -- linearised at the converged field
// by fg_solve_tangent with the derivative loads from fg_postprocess_tangent.  Responses
// keep the request order and the reference's layout (batch_response.cpp:124-369).
#include "motor.h"

#include <algorithm>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>

namespace fgcli
{
namespace
{

using fgio::MotorSampleRequest;

// One tangent direction's response (TangentRhsResponseDto).
struct TangentRhs {
  std::string name;
  std::vector<double> direction, dflux, dradial;
  double dfx = 0.0, dfy = 0.0, dtorque = 0.0;
  int32_t iterations = 0;
  double residual = std::numeric_limits<double>::infinity();
};

// One item's response (MotorBatchResponseDto without the sector fields).
struct MotorItem {
  int status = FG_INTERNAL_ERROR;
  bool tangent_requested = false;
  std::vector<double> currents, flux, angles, radial;
  int32_t iterations = 0;
  double residual = std::numeric_limits<double>::infinity();
  double fx = 0.0, fy = 0.0, torque = 0.0;
  size_t elements = 0;
  int tangent_status = FG_OK;
  std::vector<TangentRhs> rhs;
};

template <class V> void Csv(std::ostream &o, const V &v)
{
  for (size_t i = 0; i < v.size(); ++i)
    o << (i ? ", " : "") << v[i];
}

void Residual(std::ostream &o, double r)
{
  if (std::isfinite(r))
    o << r;
  else
    o << "null";
}

// WriteMotorSampleResponseJson (sample_adapter.cpp:64-123).
std::string SingleResponse(int status, const MotorSampleRequest *req, const Solved *sol, const Post *post)
{
  std::ostringstream o;
  o << std::setprecision(17) << "{\n  \"protocol\": \"" << (req ? req->protocol : "gpu_femm_motor_sample_v1")
    << "\",\n  \"mesh_artifact_sha256\": \"" << (req ? req->mesh_artifact_sha256 : "")
    << "\",\n  \"base_motor_fem_sha256\": \"" << (req ? req->base_motor_fem_sha256 : "")
    << "\",\n  \"source_fem_sha256\": \"" << (req ? req->source_fem_sha256 : "") << "\",\n"
    << "  \"status\": \"" << (status == 0 ? "PASS" : "FAIL") << "\",\n"
    << "  \"solve_status\": \"" << StatusName(status) << "\",\n"
    << "  \"error_identifier\": \"" << (status == 0 ? "" : "GPU_FEMM_" + StatusName(status)) << "\",\n"
    << "  \"error_message\": \"" << (status == 0 ? "" : StatusName(status)) << "\",\n";
  if (status == 0 && req && sol && post) {
    o << "  \"Fx_N\": " << post->fx << ",\n  \"Fy_N\": " << post->fy << ",\n  \"torque_Nm\": " << post->torque
      << ",\n  \"actual_circuit_currents_A\": [";
    Csv(o, sol->currents);
    o << "],\n  \"circuit_flux_linkage_Wb\": [";
    Csv(o, sol->flux);
    o << "],\n  \"airgap_sample_angles_deg\": [";
    Csv(o, req->airgap_angles_deg);
    o << "],\n  \"airgap_radial_flux_density_T\": [";
    Csv(o, post->radial);
    o << "],\n  \"mesh_element_count\": " << sol->b1.size() << ",\n  \"convergence\": {\"iterations\": "
      << sol->iterations << ", \"residual_l2\": " << sol->residual << "}\n";
  } else {
    o << "  \"Fx_N\": null,\n  \"Fy_N\": null,\n  \"torque_Nm\": null,\n"
      << "  \"actual_circuit_currents_A\": [],\n  \"circuit_flux_linkage_Wb\": [],\n"
      << "  \"airgap_sample_angles_deg\": [],\n  \"airgap_radial_flux_density_T\": [],\n"
      << "  \"mesh_element_count\": 0,\n  \"convergence\": {\"iterations\": " << (sol ? sol->iterations : 0)
      << ", \"residual_l2\": ";
    Residual(o, sol ? sol->residual : std::numeric_limits<double>::infinity());
    o << "}\n";
  }
  o << "}";
  return o.str();
}

// WriteMotorBatchItemResponseJson (batch_response.cpp:124-281), conforming artifacts.
void ItemResponse(std::ostream &o, const MotorSampleRequest &req, const MotorItem &d)
{
  o << std::setprecision(17) << "{\n  \"protocol\": \"" << req.protocol << "\",\n"
    << "  \"mesh_artifact_sha256\": \"" << req.mesh_artifact_sha256 << "\",\n"
    << "  \"base_motor_fem_sha256\": \"" << req.base_motor_fem_sha256 << "\",\n"
    << "  \"source_fem_sha256\": \"" << req.source_fem_sha256 << "\",\n"
    << "  \"status\": \"" << (d.status == 0 ? "PASS" : "FAIL") << "\",\n"
    << "  \"solve_status\": \"" << StatusName(d.status) << "\",\n"
    << "  \"error_identifier\": \"" << (d.status == 0 ? "" : "GPU_FEMM_" + StatusName(d.status)) << "\",\n"
    << "  \"error_message\": \"" << (d.status == 0 ? "" : StatusName(d.status)) << "\",\n";
  if (d.status == 0) {
    o << "  \"Fx_N\": " << d.fx << ",\n  \"Fy_N\": " << d.fy << ",\n  \"torque_Nm\": " << d.torque
      << ",\n  \"actual_circuit_currents_A\": [";
    Csv(o, d.currents);
    o << "],\n  \"circuit_flux_linkage_Wb\": [";
    Csv(o, d.flux);
    o << "],\n  \"airgap_sample_angles_deg\": [";
    Csv(o, d.angles);
    o << "],\n  \"airgap_radial_flux_density_T\": [";
    Csv(o, d.radial);
    o << "],\n  \"mesh_element_count\": " << d.elements << ",\n";
    if (d.tangent_requested) {
      o << "  \"tangent_multi_rhs\": {\"schema_version\": \"gpu_femm_tangent_multi_rhs_response_v1\", \"status\": \""
        << (d.tangent_status == 0 ? "PASS" : "FAIL") << "\", \"solve_status\": \"" << StatusName(d.tangent_status)
        << "\", \"error_identifier\": \"" << (d.tangent_status == 0 ? "" : "GPU_FEMM_TANGENT_" + StatusName(d.tangent_status))
        << "\", \"linearization\": \"consistent_newton_jacobian_at_converged_operating_point\", "
        << "\"base_circuit_currents_A\": [";
      Csv(o, d.currents);
      o << "], \"rhs\": [";
      for (size_t k = 0; k < d.rhs.size(); ++k) {
        const TangentRhs &r = d.rhs[k];
        o << (k ? ", " : "") << "{\"name\": \"" << r.name << "\", \"circuit_current_derivative_A_per_A\": [";
        Csv(o, r.direction);
        o << "], \"dFx_N_per_A\": " << r.dfx << ", \"dFy_N_per_A\": " << r.dfy << ", \"dtorque_Nm_per_A\": "
          << r.dtorque << ", \"circuit_flux_linkage_derivative_Wb_per_A\": [";
        Csv(o, r.dflux);
        o << "], \"airgap_radial_flux_density_derivative_T_per_A\": [";
        Csv(o, r.dradial);
        o << "], \"linear_convergence\": {\"iterations\": " << r.iterations << ", \"residual_l2\": ";
        Residual(o, r.residual);
        o << "}}";
      }
      o << "]},\n";
    }
    o << "  \"convergence\": {\"iterations\": " << d.iterations << ", \"residual_l2\": " << d.residual << "}\n";
  } else {
    o << "  \"Fx_N\": null,\n  \"Fy_N\": null,\n  \"torque_Nm\": null,\n"
      << "  \"actual_circuit_currents_A\": [],\n  \"circuit_flux_linkage_Wb\": [],\n"
      << "  \"airgap_sample_angles_deg\": [],\n  \"airgap_radial_flux_density_T\": [],\n"
      << "  \"mesh_element_count\": 0,\n  \"convergence\": {\"iterations\": " << d.iterations << ", \"residual_l2\": ";
    Residual(o, d.residual);
    o << "}\n";
  }
  o << "}";
}

// The tangent block of one solved, postprocessed item (motor_postprocess.cpp:84-183).
void Tangent(Prepared &p, fg_postprocess *pp, const MotorSampleRequest &req, const Solved &sol, MotorItem *d,
             int *launches)
{
  const size_t m = req.tangent_rhs.size(), N = sol.a.size(), E = sol.b1.size(), C = sol.currents.size();
  std::vector<double> dirs;
  for (const auto &r : req.tangent_rhs)
    dirs.insert(dirs.end(), r.second.begin(), r.second.end());
  std::vector<double> da(m * N), db1(m * E), db2(m * E), dflux(m * std::max<size_t>(C, 1));
  std::vector<fg_linear_info> info(m);
  fg_solve_options o;
  fg_production_options(&o);
  int rc = fg_solve_tangent(p.plan, sol.a.data(), sol.currents.data(), static_cast<int32_t>(m), dirs.data(), &o,
                            da.data(), db1.data(), db2.data(), dflux.data(), info.data());
  fg_timing t{};
  fg_plan_last_timing(p.plan, &t);
  *launches += static_cast<int>(t.pcg_launches);
  if (rc != 0) {
    d->tangent_status = rc;
    return;
  }
  const size_t P = static_cast<size_t>(fg_postprocess_probe_count(pp));
  std::vector<fg_postprocess_result> res(m);
  std::vector<double> radial(m * P);
  rc = fg_postprocess_tangent(pp, static_cast<int32_t>(m), sol.b1.data(), sol.b2.data(), da.data(), db1.data(),
                              db2.data(), res.data(), P ? radial.data() : nullptr);
  if (rc != 0) {
    d->tangent_status = rc;
    return;
  }
  for (size_t k = 0; k < m; ++k) {
    if (info[k].status != 0) {
      d->tangent_status = info[k].status;
      continue;
    }
    if (res[k].status != 0) {
      d->tangent_status = res[k].status;
      continue;
    }
    TangentRhs r;
    r.name = req.tangent_rhs[k].first;
    r.direction = req.tangent_rhs[k].second;
    r.dfx = res[k].force_x_n;
    r.dfy = res[k].force_y_n;
    r.dtorque = res[k].torque_nm;
    r.dflux.assign(dflux.begin() + k * C, dflux.begin() + (k + 1) * C);
    r.dradial.assign(radial.begin() + k * P, radial.begin() + (k + 1) * P);
    r.iterations = info[k].iterations;
    r.residual = info[k].residual_l2;
    d->rhs.push_back(std::move(r));
  }
  if (d->tangent_status == 0 && d->rhs.size() != m)
    d->tangent_status = FG_INTERNAL_ERROR;
}

} // namespace

int MotorSingleSample(const std::string &request_path, const std::string &response_path, const Options &opt)
{
  std::string text, error;
  MotorSampleRequest req;
  if (!ReadFile(request_path, &text) || !fgio::ParseMotorSampleRequestText(text, &req, &error)) {
    PublishAtomically(response_path, SingleResponse(FG_INVALID_ARGUMENT, nullptr, nullptr, nullptr) + "\n");
    std::cerr << "FAIL motor single-sample request: " << error << '\n';
    return 1;
  }
  Prepared p;
  Prepare(req.mesh_artifact_path, req.mesh_artifact_sha256, opt, &p);
  int status = p.status;
  error = p.error;
  if (status == 0 && !fgio::MotorRequestMatchesArtifact(req, p.artifact)) {
    status = FG_INVALID_ARGUMENT;
    error = "artifact identity, pose, or circuit-count mismatch";
  }
  const bool attempted = status == 0;
  std::vector<Solved> sols;
  Post post;
  if (attempted) {
    status = EnsurePlan(&p, opt);
    if (status == 0) {
      std::vector<int> st;
      int launches = 0;
      status = SolveCurrents(p, {&req.circuit_currents_a}, &sols, &st, &launches);
      if (status == 0)
        status = st[0];
    }
    if (status == 0) {
      fg_postprocess *pp = nullptr;
      status = p.post.Get(p.plan, req.selected_group_number, req.air_group_number, req.airgap_radius_mm,
                          req.airgap_angles_deg, &pp);
      if (status == 0)
        status = RunPost(pp, sols[0], &post);
    }
  }
  const Solved *sol = attempted && !sols.empty() ? &sols[0] : nullptr;
  if (!PublishAtomically(response_path, SingleResponse(status, &req, sol, status == 0 ? &post : nullptr) + "\n"))
    return 1;
  if (status != 0) {
    std::cerr << "FAIL motor single-sample: " << error << (error.empty() ? StatusName(status) : "") << '\n';
    return 1;
  }
  return 0;
}

std::string RunMotorBatch(const fgio::MotorBatchRequest &batch, const Options &opt, ArtifactCache *artifacts,
                          bool include_timing, std::chrono::steady_clock::time_point t0, bool *all_pass)
{
  using Clock = std::chrono::steady_clock;
  auto seconds = [](Clock::time_point a) { return std::chrono::duration<double>(Clock::now() - a).count(); };
  const double parse_s = seconds(t0);
  const size_t n = batch.items.size();
  std::vector<MotorItem> out(n);
  const int effective = std::max(1, std::min<int>(batch.max_items_per_chunk, 32));
  int cache_hits = 0, chunks = 0, launches = 0, width = 0, symbolic_hits = 0;
  double artifact_s = 0.0, solve_s = 0.0, post_s = 0.0, tangent_s = 0.0, tangent_post_s = 0.0;
  int64_t pcg_iterations = 0;
  ArtifactKey cached_operator;
  bool have_cached = false;
  for (size_t first = 0; first < n; first += effective) {
    ++chunks;
    const size_t end = std::min(n, first + static_cast<size_t>(effective));
    // Artifact gate per item, then groups of items sharing one operator, first-seen order.
    std::vector<std::pair<ArtifactKey, std::vector<size_t>>> groups;
    const auto a0 = Clock::now();
    for (size_t i = first; i < end; ++i) {
      const MotorSampleRequest &r = batch.items[i].request;
      const ArtifactKey key{r.mesh_artifact_path, r.mesh_artifact_sha256};
      std::shared_ptr<Prepared> &slot = (*artifacts)[key];
      if (!slot) {
        slot = std::make_shared<Prepared>();
        Prepare(key.first, key.second, opt, slot.get());
      }
      out[i].tangent_requested = r.tangent_requested;
      out[i].status = slot->status;
      if (out[i].status != 0)
        continue;
      if (!fgio::MotorRequestMatchesArtifact(r, slot->artifact)) {
        out[i].status = FG_INVALID_ARGUMENT;
        continue;
      }
      auto g = std::find_if(groups.begin(), groups.end(), [&](const auto &x) { return x.first == key; });
      if (g == groups.end())
        groups.push_back({key, {i}});
      else
        g->second.push_back(i);
    }
    artifact_s += seconds(a0);
    for (auto &g : groups) {
      Prepared &p = *(*artifacts)[g.first];
      const std::vector<size_t> &idx = g.second;
      const int plan_status = EnsurePlan(&p, opt);
      if (plan_status != 0) {
        for (size_t i : idx)
          out[i].status = plan_status;
        have_cached = false;
        continue;
      }
      if (have_cached && cached_operator == g.first) {
        cache_hits += static_cast<int>(idx.size());
      } else {
        cache_hits += static_cast<int>(idx.size()) - 1;
        cached_operator = g.first;
        have_cached = true;
      }
      width = std::max(width, static_cast<int>(idx.size()));
      std::vector<const std::vector<double> *> currents;
      for (size_t i : idx)
        currents.push_back(&batch.items[i].request.circuit_currents_a);
      std::vector<Solved> sols;
      std::vector<int> st;
      const auto s0 = Clock::now();
      SolveCurrents(p, currents, &sols, &st, &launches);
      solve_s += seconds(s0);
      fg_timing t{};
      fg_plan_last_timing(p.plan, &t);
      pcg_iterations += t.pcg_iterations;
      for (size_t j = 0; j < idx.size(); ++j) {
        const size_t i = idx[j];
        const MotorSampleRequest &r = batch.items[i].request;
        MotorItem &d = out[i];
        d.status = st[j];
        if (!sols.empty()) {
          d.currents = sols[j].currents;
          d.iterations = sols[j].iterations;
          d.residual = sols[j].residual;
        }
        if (d.status != 0)
          continue;
        const auto p0 = Clock::now();
        fg_postprocess *pp = nullptr;
        Post post;
        d.status = p.post.Get(p.plan, r.selected_group_number, r.air_group_number, r.airgap_radius_mm,
                              r.airgap_angles_deg, &pp);
        if (d.status == 0)
          d.status = RunPost(pp, sols[j], &post);
        post_s += seconds(p0);
        if (d.status != 0)
          continue;
        d.fx = post.fx;
        d.fy = post.fy;
        d.torque = post.torque;
        d.flux = sols[j].flux;
        d.angles = r.airgap_angles_deg;
        d.radial = post.radial;
        d.elements = sols[j].b1.size();
        if (r.tangent_requested) {
          const auto q0 = Clock::now();
          Tangent(p, pp, r, sols[j], &d, &launches);
          tangent_s += seconds(q0);
          ++symbolic_hits; // the tangent operator reuses the plan's symbolic CSR
        }
      }
    }
  }
  bool pass = true;
  for (const MotorItem &d : out)
    pass = pass && d.status == 0;
  *all_pass = pass;
  std::ostringstream o;
  o << std::setprecision(17) << "{\n  \"protocol\": \"" << batch.protocol << "\",\n"
    << "  \"status\": \"" << (pass ? "PASS" : "FAIL") << "\",\n"
    << "  \"solve_status\": \"" << (pass ? "PASS" : "PARTIAL_FAILURE") << "\",\n"
    << "  \"error_identifier\": \"" << (pass ? "" : "GPU_FEMM_BATCH_PARTIAL_FAILURE") << "\",\n"
    << "  \"error_message\": \"" << (pass ? "" : "one or more batch items failed") << "\",\n"
    << "  \"cache\": {\"mesh_cache_hits\": " << cache_hits << ", \"chunk_count\": " << chunks
    << ", \"requested_chunk_size\": " << batch.max_items_per_chunk << ", \"effective_chunk_size\": " << effective
    << ", \"actual_parallel_width\": " << width << ", \"csr_symbolic_cache_hits\": " << symbolic_hits
    << ", \"batched_pcg_launches\": " << launches << "},\n";
  if (include_timing) {
    const double total = seconds(t0);
    // The reference's timing schema; phases this solver does not have report zero.
    o << "  \"timing\": {\"schema_version\": \"gpu_femm_motor_batch_timing_v1\", \"request_read_parse_seconds\": "
      << parse_s << ", \"preflight_seconds\": 0, \"artifact_read_validate_seconds\": " << artifact_s
      << ", \"solver_initialize_seconds\": 0, \"nonlinear_prepare_compute_seconds\": 0"
      << ", \"nonlinear_prepare_wait_seconds\": 0, \"host_assembly_seconds\": 0, \"device_assembly_seconds\": 0"
      << ", \"gpu_upload_seconds\": 0, \"gpu_kernel_sync_seconds\": " << solve_s
      << ", \"gpu_download_seconds\": 0, \"linear_solver\": \"pcg\", \"direct_analyses\": 0"
      << ", \"direct_factorizations\": 0, \"direct_solves\": 0, \"direct_parallel_batches\": 0"
      << ", \"direct_peak_parallel_width\": 0, \"direct_ordering_reuses\": 0, \"direct_factor_reuses\": 0"
      << ", \"direct_analysis_seconds\": 0, \"direct_factor_seconds\": 0, \"direct_solve_seconds\": 0"
      << ", \"direct_peak_plan_device_bytes\": 0, \"preconditioner\": \""
      << (opt.plan.preconditioner == FG_PRECOND_JACOBI ? "jacobi" : "block-jacobi")
      << "\", \"preconditioner_setup_seconds\": 0, \"interleaved_spmv_solves\": 0, \"preconditioner_builds\": 0"
      << ", \"preconditioner_block_size\": "
      << (opt.plan.preconditioner == FG_PRECOND_JACOBI ? 1 : opt.plan.block_size)
      << ", \"nonlinear_pcg_iterations\": " << pcg_iterations
      << ", \"preconditioner_reuses\": 0, \"preconditioner_fallback_blocks\": 0, \"state_update_seconds\": 0"
      << ", \"finalize_seconds\": 0, \"nonlinear_recovery_seconds\": 0, \"postprocess_plan_compute_seconds\": 0"
      << ", \"postprocess_plan_seconds\": 0, \"base_postprocess_seconds\": " << post_s
      << ", \"tangent_operator_seconds\": " << tangent_s << ", \"tangent_postprocess_seconds\": " << tangent_post_s
      << ", \"postprocess_seconds\": " << post_s + tangent_s
      << ", \"measured_before_response_write_seconds\": " << total << "},\n";
  }
  o << "  \"items\": [\n";
  for (size_t i = 0; i < n; ++i) {
    o << "    {\"task_id\": \"" << batch.items[i].task_id << "\", \"response\": ";
    ItemResponse(o, batch.items[i].request, out[i]);
    o << "}" << (i + 1 == n ? "\n" : ",\n");
  }
  o << "  ]\n}\n";
  return o.str();
}

int MotorBatch(const std::string &request_path, const std::string &response_path, const Options &opt,
               bool include_timing)
{
  const auto t0 = std::chrono::steady_clock::now();
  std::string text, error;
  fgio::MotorBatchRequest batch;
  if (!ReadFile(request_path, &text) || !fgio::ParseMotorBatchRequestText(text, &batch, &error)) {
    // No trusted item identity exists to write a resumable response.
    std::cerr << "FAIL motor batch request: " << error << '\n';
    return 1;
  }
  ArtifactCache artifacts;
  bool pass = false;
  const std::string body = RunMotorBatch(batch, opt, &artifacts, include_timing, t0, &pass);
  if (!PublishAtomically(response_path, body))
    return 1;
  return pass ? 0 : 1;
}

} // namespace fgcli
