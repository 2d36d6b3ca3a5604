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
  // gpu_femm_motor_sample_v3 on a sector: the full-machine reconstruction.
  bool sector = false;
  int sector_status = FG_OK;
  int base_sign = 1, tangent_sign = 1;
  double base_torque_multiplier = 2.0, tangent_force_multiplier = 0.0, tangent_torque_multiplier = 0.0;
  size_t evidence_operators = 0, evidence_uploads = 0, evidence_rhs = 0, evidence_operator_bytes = 0,
         evidence_rhs_bytes = 0;
};

// MapSectorAirgapAnglesToRepresentative (sample_request.cpp:531-558): probes folded into the
// half-turn that starts at the sector start; odd copies take the repeat sign.
std::vector<int> FoldSectorAngles(double start_rad, int repeat_sign, std::vector<double> *angles)
{
  std::vector<int> signs;
  for (double &angle : *angles) {
    int64_t copy = static_cast<int64_t>(std::floor((angle - start_rad) / kPi));
    angle -= static_cast<double>(copy) * kPi;
    const double tol = 64.0 * std::numeric_limits<double>::epsilon() *
                       std::max({1.0, std::abs(angle), std::abs(start_rad)});
    if (angle < start_rad - tol) {
      angle += kPi;
      --copy;
    } else if (angle >= start_rad + kPi - tol) {
      angle -= kPi;
      ++copy;
    }
    if (std::abs(angle - start_rad) <= tol)
      angle = start_rad;
    signs.push_back(std::abs(copy) % 2 != 0 ? repeat_sign : 1);
  }
  return signs;
}

// ReconstructSectorCircuitFluxLinkage (batch_response.cpp:20-35): each circuit's flux plus its
// partner copy's, oriented and signed by the field's repeat relation.
std::vector<double> ReconstructFlux(const std::vector<double> &sector, const fgio::Artifact &a, int sign)
{
  if (sector.size() != a.circuit_partners.size())
    return {};
  std::vector<double> full = sector;
  for (size_t c = 0; c < sector.size(); ++c)
    full[a.circuit_partners[c]] += static_cast<double>(a.circuit_orientations[c] * sign) * sector[c];
  return full;
}

// MapNativeAgeSectorAirgapAnglesToRepresentative (sample_request.cpp:568-599): a native
// air-gap element sector's series is referenced to angle 0, so probes fold into [0, span);
// odd copies of an antiperiodic sector take the sign -1.
std::vector<int> FoldNativeSectorAngles(double span, int boundary_sign, std::vector<double> *angles)
{
  std::vector<int> signs;
  for (double &angle : *angles) {
    int64_t copy = static_cast<int64_t>(std::floor(angle / span));
    double local = angle - static_cast<double>(copy) * span;
    const double tol = 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::abs(local));
    if (local < -tol) {
      local += span;
      --copy;
    } else if (local >= span - tol) {
      local -= span;
      ++copy;
    }
    if (std::abs(local) <= tol)
      local = 0.0;
    angle = local;
    signs.push_back(std::abs(copy) % 2 != 0 && boundary_sign < 0 ? -1 : 1);
  }
  return signs;
}

// ReconstructCyclicSectorCircuitFluxLinkage (batch_response.cpp:38-55): each circuit's sector
// flux lands on the circuits its k copies become, with the partner orientation and the
// boundary relation's sign accumulated copy by copy.
std::vector<double> ReconstructCyclicFlux(const std::vector<double> &sector, const fgio::Artifact &a)
{
  if (sector.size() != a.circuit_partners.size() || sector.size() != a.circuit_orientations.size())
    return {};
  std::vector<double> full(sector.size(), 0.0);
  for (size_t c = 0; c < sector.size(); ++c) {
    int32_t at = static_cast<int32_t>(c);
    int sign = 1;
    for (int32_t copy = 0; copy < a.full_machine_sector_count; ++copy) {
      full[at] += static_cast<double>(sign) * sector[c];
      sign *= a.circuit_orientations[at] * a.sector_boundary_sign;
      at = a.circuit_partners[at];
    }
  }
  return full;
}

// MakeMotorSectorTangentModel (sample_request.cpp:499-529): the suspension order's boundary
// relation on every pair; apex nodes fixed to zero only when that relation is antiperiodic.
int SectorTangentPlan(Prepared &p, const Options &opt)
{
  if (p.sector_tangent_tried)
    return p.sector_tangent ? p.sector_tangent->plan_status : FG_INVALID_ARGUMENT;
  p.sector_tangent_tried = true;
  auto t = std::make_shared<Prepared>();
  t->artifact = p.artifact;
  fgio::Artifact &a = t->artifact;
  const int sign = a.suspension_spatial_order % 2 == 0 ? 1 : -1;
  for (int32_t apex : a.apex_nodes)
    for (size_t i = 0; i < a.dir_nodes.size();) {
      if (a.dir_nodes[i] == apex) {
        a.dir_nodes.erase(a.dir_nodes.begin() + i);
        a.dir_values.erase(a.dir_values.begin() + i);
      } else {
        ++i;
      }
    }
  if (sign < 0)
    for (int32_t apex : a.apex_nodes) {
      a.dir_nodes.push_back(apex);
      a.dir_values.push_back(0.0);
    }
  for (int8_t &s : a.con_signs)
    s = static_cast<int8_t>(sign);
  const int rc = EnsurePlan(t.get(), opt);
  if (rc != 0)
    return FG_INVALID_ARGUMENT; // the tangent model failed validation
  p.sector_tangent = t;
  return 0;
}

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

// The sector_reconstruction member (batch_response.cpp:164-222), conforming sectors.
void SectorBlock(std::ostream &o, const MotorItem &d, const fgio::Artifact &a)
{
  const bool native = a.sliding_band;
  o << "  \"sector_reconstruction\": {\"schema_version\": "
    << (native ? "\"gpu_femm_motor_sector_reconstruction_v2\", " : "\"gpu_femm_motor_sector_reconstruction_response_v1\", ")
    << "\"status\": \"" << (d.sector_status == 0 ? "PASS" : "FAIL") << "\", \"error_identifier\": \""
    << (d.sector_status == 0 ? "" : "GPU_FEMM_SECTOR_" + StatusName(d.sector_status))
    << "\", \"sector_start_angle_deg\": " << a.sector_start_angle_deg << ", \"sector_angle_deg\": " << a.sector_angle_deg
    << ", \"full_machine_sector_count\": " << a.full_machine_sector_count
    << ", \"electrical_pole_pairs\": " << a.electrical_pole_pairs
    << ", \"suspension_spatial_order\": " << a.suspension_spatial_order << ", \"base_boundary_relation\": \""
    << (d.base_sign > 0 ? "periodic" : "antiperiodic") << "\", \"tangent_boundary_relation\": \""
    << (d.tangent_sign > 0 ? "periodic" : "antiperiodic") << "\", \"base_field_repeat_sign\": " << d.base_sign
    << ", \"tangent_field_repeat_sign\": " << d.tangent_sign << ", \"output_normalization\": \"full_machine\""
    << ", \"load_extraction_method\": \""
    << (native ? "native_air_gap_element_signed_sector" : "weighted_stress_tensor_periodic_pair_mask")
    << "\", \"periodic_pair_aware_weighted_stress_mask\": " << (native ? "false" : "true")
    << ", \"constraint_source\": \"cropped_sector_artifact\", \"operator_construction\": \""
    << (native ? "native_age_sector_base_only" : "same_topology_dual_signed_reduction") << "\""
    << ", \"tangent_operator_storage\": \"shared_single_upload\", \"tangent_physical_operator_count\": "
    << d.evidence_operators << ", \"tangent_operator_upload_count\": " << d.evidence_uploads
    << ", \"tangent_rhs_count\": " << d.evidence_rhs << ", \"tangent_operator_bytes\": " << d.evidence_operator_bytes
    << ", \"tangent_rhs_workspace_bytes\": " << d.evidence_rhs_bytes
    << ", \"base_force_rule\": \"sum_rotated_sector_vectors\", \"base_torque_multiplier\": "
    << d.base_torque_multiplier << ", \"tangent_force_multiplier\": " << d.tangent_force_multiplier
    << ", \"tangent_torque_multiplier\": " << d.tangent_torque_multiplier << ", \"circuit_partner_indices\": [";
  Csv(o, a.circuit_partners);
  o << "], \"circuit_partner_orientations\": [";
  for (size_t i = 0; i < a.circuit_orientations.size(); ++i)
    o << (i ? ", " : "") << static_cast<int>(a.circuit_orientations[i]);
  o << "], \"apex_self_pair_nodes\": [";
  Csv(o, a.apex_nodes);
  o << "], \"model_invariance_certificate_sha256\": \"" << a.model_invariance_certificate_sha256 << "\"},\n";
}

// WriteMotorBatchItemResponseJson (batch_response.cpp:124-281), conforming artifacts.
void ItemResponse(std::ostream &o, const MotorSampleRequest &req, const MotorItem &d, const fgio::Artifact *art)
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
    if (d.sector && art)
      SectorBlock(o, d, *art);
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
void Tangent(fg_plan *plan, fg_postprocess *pp, const MotorSampleRequest &req, const Solved &sol, MotorItem *d,
             int *launches, const std::vector<int> *radial_signs = nullptr)
{
  const size_t m = req.tangent_rhs.size(), N = sol.a.size(), E = sol.b1.size(), C = sol.currents.size();
  std::vector<double> dirs;
  for (const auto &r : req.tangent_rhs)
    dirs.insert(dirs.end(), r.second.begin(), r.second.end());
  std::vector<double> da(m * N), db1(m * E), db2(m * E), dflux(m * std::max<size_t>(C, 1));
  std::vector<fg_linear_info> info(m);
  fg_solve_options o;
  fg_production_options(&o);
  int rc = fg_solve_tangent(plan, sol.a.data(), sol.currents.data(), static_cast<int32_t>(m), dirs.data(), &o,
                            da.data(), db1.data(), db2.data(), dflux.data(), info.data());
  fg_timing t{};
  fg_plan_last_timing(plan, &t);
  *launches += static_cast<int>(t.pcg_launches);
  if (rc != 0) {
    d->tangent_status = rc;
    return;
  }
  // pp null: a sliding-band plan, whose derivatives come from its air-gap elements
  // (ComputeAirGapElementTangentPostprocess) at the request's probe angles.
  std::vector<double> angles;
  for (double deg : req.airgap_angles_deg)
    angles.push_back(deg * kPi / 180.0);
  const size_t P = pp ? static_cast<size_t>(fg_postprocess_probe_count(pp)) : angles.size();
  std::vector<fg_postprocess_result> res(m);
  std::vector<double> radial(m * P);
  rc = pp ? fg_postprocess_tangent(pp, static_cast<int32_t>(m), sol.b1.data(), sol.b2.data(), da.data(),
                                   db1.data(), db2.data(), res.data(), P ? radial.data() : nullptr)
          : fg_air_gap_tangent(plan, static_cast<int32_t>(m), sol.a.data(), da.data(),
                               static_cast<int32_t>(P), P ? angles.data() : nullptr, res.data(),
                               P ? radial.data() : nullptr);
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
    if (radial_signs)
      for (size_t j = 0; j < P && j < radial_signs->size(); ++j)
        r.dradial[j] *= (*radial_signs)[j];
    r.iterations = info[k].iterations;
    r.residual = info[k].residual_l2;
    d->rhs.push_back(std::move(r));
  }
  if (d->tangent_status == 0 && d->rhs.size() != m)
    d->tangent_status = FG_INTERNAL_ERROR;
}

// The samples of a chunk's operators -- motor artifacts, and the poses of sliding-band
// artifacts -- in one multi-plan launch per Newton step (SolveOperatorsTogether); false
// when that does not apply (then the caller solves operator by operator).
// pre[item] = (solution, status).
template <class Groups>
bool MultiSolvePoses(const Groups &groups, const fgio::MotorBatchRequest &batch, const Options &opt,
                     ArtifactCache *artifacts, std::map<size_t, std::pair<Solved, int>> *pre, int *launches,
                     int64_t *pcg_iterations)
{
  std::vector<Operator> ops;
  for (const auto &g : groups) {
    Prepared &base = *(*artifacts)[g.first.first];
    if (base.status != 0)
      return false;
    Operator op{PoseOf(base, g.first.second), {}};
    for (size_t i : g.second)
      op.currents.push_back(&batch.items[i].request.circuit_currents_a);
    ops.push_back(std::move(op));
  }
  std::vector<std::vector<Solved>> sols;
  std::vector<std::vector<int>> st;
  if (!SolveOperatorsTogether(ops, opt, &sols, &st, launches, pcg_iterations))
    return false;
  size_t o = 0;
  for (const auto &g : groups) {
    for (size_t j = 0; j < g.second.size(); ++j)
      (*pre)[g.second[j]] = {std::move(sols[o][j]), st[o][j]};
    ++o;
  }
  return true;
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
  Prepared &q = status == 0 ? *PoseOf(p, req.rotor_angle_deg) : p;
  if (status == 0 && q.status != 0) {
    status = q.status;
    error = q.error;
  }
  const bool attempted = status == 0;
  std::vector<Solved> sols;
  Post post;
  if (attempted) {
    status = EnsurePlan(&q, opt);
    if (status == 0) {
      std::vector<int> st;
      int launches = 0;
      status = SolveCurrents(q, {&req.circuit_currents_a}, &sols, &st, &launches);
      if (status == 0)
        status = st[0];
    }
    if (status == 0 && q.artifact.sliding_band) {
      status = AirGapPost(q.plan, sols[0], req.airgap_angles_deg, &post);
    } else if (status == 0) {
      fg_postprocess *pp = nullptr;
      status = q.post.Get(q.plan, req.selected_group_number, req.air_group_number, req.airgap_radius_mm,
                          req.airgap_angles_deg, &pp, nullptr, &q.artifact.apex_nodes);
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
  // An operator is an artifact, and for a sliding-band artifact also the rotor angle
  // (MotorBatchOperatorKey, batch_prepare.cpp:220-233).
  using OperatorKey = std::pair<ArtifactKey, double>;
  OperatorKey cached_operator;
  bool have_cached = false;
  for (size_t first = 0; first < n; first += effective) {
    ++chunks;
    for (auto &kv : *artifacts)
      if (kv.second)
        TrimPoses(*kv.second, kResidentPoses);
    const size_t end = std::min(n, first + static_cast<size_t>(effective));
    // Artifact gate per item, then groups of items sharing one operator, first-seen order.
    std::vector<std::pair<OperatorKey, std::vector<size_t>>> groups;
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
      const OperatorKey op{key, slot->artifact.sliding_band ? r.rotor_angle_deg : 0.0};
      const Prepared *pose = PoseOf(*slot, r.rotor_angle_deg);
      if (pose->status != 0) {
        out[i].status = pose->status;
        continue;
      }
      auto g = std::find_if(groups.begin(), groups.end(), [&](const auto &x) { return x.first == op; });
      if (g == groups.end())
        groups.push_back({op, {i}});
      else
        g->second.push_back(i);
    }
    artifact_s += seconds(a0);
    std::map<size_t, std::pair<Solved, int>> pre;
    {
      const auto m0 = Clock::now();
      MultiSolvePoses(groups, batch, opt, artifacts, &pre, &launches, &pcg_iterations);
      solve_s += seconds(m0);
    }
    for (auto &g : groups) {
      Prepared &p = *PoseOf(*(*artifacts)[g.first.first], g.first.second);
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
      if (pre.count(idx[0])) {
        for (size_t i : idx) {
          sols.push_back(pre[i].first);
          st.push_back(pre[i].second);
        }
      } else {
        const auto s0 = Clock::now();
        SolveCurrents(p, currents, &sols, &st, &launches);
        solve_s += seconds(s0);
        fg_timing t{};
        fg_plan_last_timing(p.plan, &t);
        pcg_iterations += t.pcg_iterations;
      }
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
        const bool sector = r.sector_performance && p.artifact.sector;
        std::vector<int> base_signs, tangent_signs;
        std::vector<double> folded;
        const bool native = sector && p.artifact.native_sector;
        if (sector) {
          for (double deg : r.airgap_angles_deg)
            folded.push_back(deg * kPi / 180.0);
          std::vector<double> tangent_folded = folded;
          const double start = p.artifact.sector_start_angle_deg * kPi / 180.0;
          d.base_sign = p.artifact.sector_boundary_sign;
          d.tangent_sign = p.artifact.suspension_spatial_order % 2 == 0 ? 1 : -1;
          if (native) {
            base_signs = FoldNativeSectorAngles(p.artifact.sector_angle_deg * kPi / 180.0, d.base_sign, &folded);
          } else {
            base_signs = FoldSectorAngles(start, d.base_sign, &folded);
            tangent_signs = FoldSectorAngles(start, d.tangent_sign, &tangent_folded);
          }
        }
        if (p.artifact.sliding_band) {
          d.status = AirGapPost(p.plan, sols[j], r.airgap_angles_deg, &post, native ? &folded : nullptr);
        } else {
          d.status = p.post.Get(p.plan, r.selected_group_number, r.air_group_number, r.airgap_radius_mm,
                                r.airgap_angles_deg, &pp, sector ? &folded : nullptr, &p.artifact.apex_nodes);
          if (d.status == 0)
            d.status = RunPost(pp, sols[j], &post);
        }
        post_s += seconds(p0);
        if (d.status == 0 && sector)
          for (size_t k = 0; k < post.radial.size() && k < base_signs.size(); ++k)
            post.radial[k] *= base_signs[k];
        if (d.status == 0) {
          d.fx = post.fx;
          d.fy = post.fy;
          d.torque = post.torque;
          d.flux = sols[j].flux;
          d.angles = r.airgap_angles_deg;
          d.radial = post.radial;
          d.elements = sols[j].b1.size();
        }
        if (sector) {
          // ApplyBaseSectorReconstruction (batch_response.cpp:56-99): the orbit cancels the
          // force, doubles the torque, and the partner circuits complete the flux.
          d.sector = true;
          const int cross = d.base_sign * d.tangent_sign;
          d.tangent_force_multiplier = 1.0 - cross;
          d.tangent_torque_multiplier = 1.0 + cross;
          d.base_torque_multiplier = native ? static_cast<double>(p.artifact.full_machine_sector_count) : 2.0;
          if (d.status == 0) {
            d.fx = 0.0;
            d.fy = 0.0;
            d.torque *= d.base_torque_multiplier;
            d.flux = native ? ReconstructCyclicFlux(d.flux, p.artifact) : ReconstructFlux(d.flux, p.artifact, d.base_sign);
            if (d.flux.empty())
              d.status = FG_INTERNAL_ERROR;
          }
          d.sector_status = d.status;
        }
        if (d.status != 0 || !r.tangent_requested)
          continue;
        const auto q0 = Clock::now();
        d.tangent_status = 0;
        fg_plan *tangent_plan = p.plan;
        if (sector) {
          d.tangent_status = SectorTangentPlan(p, opt);
          tangent_plan = d.tangent_status == 0 ? p.sector_tangent->plan : nullptr;
        }
        if (d.tangent_status == 0) {
          Tangent(tangent_plan, pp, r, sols[j], &d, &launches, sector ? &tangent_signs : nullptr);
          ++symbolic_hits; // the tangent operator reuses a resident symbolic CSR
          if (sector) {
            fg_plan_sizes z{};
            fg_plan_sizes_get(tangent_plan, &z);
            const size_t m = r.tangent_rhs.size();
            d.evidence_operators = d.evidence_uploads = 1;
            d.evidence_rhs = m;
            d.evidence_operator_bytes = static_cast<size_t>(z.nnz + 2 * z.rows) * sizeof(double);
            d.evidence_rhs_bytes = m * static_cast<size_t>(z.rows) * 7 * sizeof(double) + m * sizeof(fg_linear_info);
          }
        }
        if (sector) {
          // ApplyTangentSectorReconstruction (batch_response.cpp:101-113).
          for (TangentRhs &t : d.rhs) {
            t.dfx *= d.tangent_force_multiplier;
            t.dfy *= d.tangent_force_multiplier;
            t.dtorque *= d.tangent_torque_multiplier;
            t.dflux = ReconstructFlux(t.dflux, p.artifact, d.tangent_sign);
            if (t.dflux.empty())
              d.tangent_status = FG_INTERNAL_ERROR;
          }
          d.sector_status = d.tangent_status;
        }
        tangent_s += seconds(q0);
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
    const MotorSampleRequest &r = batch.items[i].request;
    auto it = artifacts->find({r.mesh_artifact_path, r.mesh_artifact_sha256});
    ItemResponse(o, r, out[i], it != artifacts->end() && it->second ? &it->second->artifact : nullptr);
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
