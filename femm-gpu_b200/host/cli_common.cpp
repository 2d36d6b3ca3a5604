// cli_common.cpp -- pieces shared by the femm_gpu adapters.
#include "cli_common.h"

#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace fgcli
{

std::string StatusName(int s) { return fg_status_name(s); }

bool ReadFile(const std::string &path, std::string *out)
{
  std::ifstream f(path, std::ios::binary);
  if (!f)
    return false;
  std::stringstream ss;
  ss << f.rdbuf();
  *out = ss.str();
  return static_cast<bool>(f) || f.eof();
}

bool SameFile(const std::string &a, const std::string &b)
{
  struct stat sa {}, sb {};
  if (stat(a.c_str(), &sa) == 0 && stat(b.c_str(), &sb) == 0)
    return sa.st_dev == sb.st_dev && sa.st_ino == sb.st_ino;
  char ra[4096], rb[4096];
  const char *pa = realpath(a.c_str(), ra), *pb = realpath(b.c_str(), rb);
  return std::string(pa ? pa : a.c_str()) == std::string(pb ? pb : b.c_str());
}

bool PublishAtomically(const std::string &path, const std::string &text)
{
  static std::atomic<uint64_t> sequence{0};
  const std::string tmp = path + ".tmp." +
                          std::to_string(std::chrono::steady_clock::now().time_since_epoch().count()) +
                          "." + std::to_string(sequence.fetch_add(1));
  {
    std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
    if (!f)
      return false;
    f << text;
    f.flush();
    if (!f) {
      std::remove(tmp.c_str());
      return false;
    }
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) {
    std::remove(tmp.c_str());
    return false;
  }
  return true;
}

// The postprocess options of an adapter request (sample_adapter.cpp:51-58, :426-432):
// group selection, a mask PCG of at most 4096 iterations, the circle in metres and radians.
fg_postprocess_options PostOptions(int32_t selected_group, int32_t air_group, double radius_mm,
                                   const std::vector<double> &angles_deg, std::vector<double> *angles)
{
  fg_postprocess_options o;
  fg_postprocess_default_options(&o);
  o.selected_group_number = selected_group;
  o.air_group_number = air_group;
  o.max_mask_iterations = 4096;
  o.airgap_radius_m = radius_mm * 1e-3;
  angles->clear();
  for (double deg : angles_deg)
    angles->push_back(deg * kPi / 180.0);
  o.airgap_angle_count = static_cast<int32_t>(angles->size());
  o.airgap_angles_rad = angles->data();
  return o;
}

int RunPost(fg_postprocess *pp, const Solved &s, Post *out)
{
  fg_postprocess_result r{};
  out->radial.assign(static_cast<size_t>(fg_postprocess_probe_count(pp)), 0.0);
  const int rc = fg_postprocess_compute(pp, 1, s.a.data(), s.b1.data(), s.b2.data(), &r, out->radial.data());
  if (rc != 0)
    return rc;
  out->fx = r.force_x_n;
  out->fy = r.force_y_n;
  out->torque = r.torque_nm;
  return r.status;
}

Prepared *PoseOf(Prepared &p, double rotor_angle_deg)
{
  if (p.status != 0 || !p.artifact.sliding_band)
    return &p;
  std::shared_ptr<Prepared> &slot = p.poses[rotor_angle_deg];
  if (!slot) {
    slot = std::make_shared<Prepared>();
    slot->artifact = p.artifact;
    if (!slot->artifact.SlideBands(rotor_angle_deg)) {
      slot->status = FG_INVALID_ARGUMENT;
      slot->error = "could not apply the requested sliding-band angle";
    }
  }
  slot->last_use = ++p.pose_clock;
  return slot.get();
}

void TrimPoses(Prepared &p, size_t keep)
{
  while (p.poses.size() > keep) {
    auto oldest = p.poses.begin();
    for (auto it = p.poses.begin(); it != p.poses.end(); ++it)
      if (it->second->last_use < oldest->second->last_use)
        oldest = it;
    p.poses.erase(oldest);
  }
}

int AirGapPost(fg_plan *plan, const Solved &s, const std::vector<double> &angles_deg, Post *out,
               const std::vector<double> *angles_rad)
{
  std::vector<double> angles;
  for (double deg : angles_deg)
    angles.push_back(deg * kPi / 180.0);
  if (angles_rad)
    angles = *angles_rad;
  out->radial.assign(angles.size(), 0.0);
  fg_postprocess_result r{};
  const int rc = fg_air_gap_postprocess(plan, 1, s.a.data(), static_cast<int32_t>(angles.size()),
                                        angles.empty() ? nullptr : angles.data(), &r,
                                        angles.empty() ? nullptr : out->radial.data());
  if (rc != 0)
    return rc;
  out->fx = r.force_x_n;
  out->fy = r.force_y_n;
  out->torque = r.torque_nm;
  return r.status;
}

void Prepare(const std::string &path, const std::string &sha, const Options &opt, Prepared *p)
{
  std::string bytes;
  if (!ReadFile(path, &bytes)) {
    p->status = FG_INPUT_IO;
    p->error = "cannot open mesh artifact";
  } else if (fgio::Sha256Hex(bytes) != sha) {
    p->status = FG_INVALID_ARGUMENT;
    p->error = "mesh artifact SHA mismatch";
  } else if (!fgio::ParseArtifact(bytes, &p->artifact, &p->error)) {
    p->status = FG_INVALID_ARGUMENT;
  }
}

void PreparePlanOnHost(Prepared *p, const Options &opt)
{
  if (p->status != 0 || p->plan_status >= 0)
    return;
  fg_model m = p->artifact.Model();
  fg_plan_options o = opt.plan;
  o.flags |= FG_PLAN_HOST_ONLY;
  p->plan_status = fg_plan_create(&m, &o, &p->plan);
  if (p->plan_status != 0)
    p->plan = nullptr;
  p->host_only = p->plan_status == 0;
}

int EnsurePlan(Prepared *p, const Options &opt)
{
  if (p->plan && p->host_only) {
    const int rc = fg_plan_attach_device(p->plan);
    if (rc != 0)
      return rc;
    p->host_only = false;
  }
  if (p->plan)
    return 0;
  if (p->plan_status > 0)
    return p->plan_status;
  fg_model m = p->artifact.Model();
  const int rc = fg_plan_create(&m, &opt.plan, &p->plan);
  if (rc != 0)
    p->plan = nullptr;
  p->plan_status = rc;
  return rc;
}

bool SolveOperatorsTogether(const std::vector<Operator> &ops, const Options &opt,
                            std::vector<std::vector<Solved>> *out, std::vector<std::vector<int>> *statuses,
                            int *launches, int64_t *pcg_iterations)
{
  if (opt.plan.preconditioner != FG_PRECOND_JACOBI || opt.plan.precision != FG_PRECISION_FP64 ||
      (opt.plan.flags & FG_PLAN_PCG_FROM_ITERATE) || ops.size() < 2)
    return false;
  for (const Operator &op : ops)
    if (!op.p || op.p->status != 0 || op.currents.empty() || op.currents.size() > kMultiGroupItems)
      return false;
  // Replica plans live only for this solve: a resident artifact keeps just its own plan,
  // so a long-running worker's device memory does not grow with the batches it has served.
  struct ReplicaPlans {
    std::vector<fg_plan *> plans;
    ~ReplicaPlans()
    {
      for (fg_plan *r : plans)
        fg_plan_destroy(r);
    }
  } replicas;
  std::vector<fg_plan *> plans;
  std::vector<std::pair<size_t, size_t>> where; // (operator, sample) of each plan
  for (size_t o = 0; o < ops.size(); ++o) {
    Prepared &p = *ops[o].p;
    if (EnsurePlan(&p, opt) != 0)
      return false;
    fg_model m = p.artifact.Model();
    for (size_t j = 0; j < ops[o].currents.size(); ++j) {
      fg_plan *plan = p.plan;
      if (j > 0) {
        plan = nullptr;
        if (fg_plan_create(&m, &opt.plan, &plan) != 0)
          return false;
        replicas.plans.push_back(plan);
      }
      plans.push_back(plan);
      where.push_back({o, j});
    }
  }
  fg_multi *multi = nullptr;
  if (fg_multi_create(plans.data(), static_cast<int32_t>(plans.size()), &multi) != 0)
    return false;
  out->assign(ops.size(), {});
  statuses->assign(ops.size(), {});
  for (size_t o = 0; o < ops.size(); ++o) {
    (*out)[o].resize(ops[o].currents.size());
    (*statuses)[o].assign(ops[o].currents.size(), FG_INTERNAL_ERROR);
  }
  const size_t M = plans.size();
  std::vector<const double *> cur(M);
  std::vector<double *> a(M), b1(M), b2(M), flux(M);
  for (size_t i = 0; i < M; ++i) {
    const Operator &op = ops[where[i].first];
    const fg_model m = op.p->artifact.Model();
    Solved &s = (*out)[where[i].first][where[i].second];
    s.currents = *op.currents[where[i].second];
    s.a.assign(m.node_count, 0.0);
    s.b1.assign(m.triangle_count, 0.0);
    s.b2.assign(m.triangle_count, 0.0);
    s.flux.assign(m.circuit_count, 0.0);
    cur[i] = s.currents.data();
    a[i] = s.a.data();
    b1[i] = s.b1.data();
    b2[i] = s.b2.data();
    flux[i] = s.flux.data();
  }
  std::vector<fg_item_info> info(M);
  fg_solve_options o;
  fg_production_options(&o);
  const int rc = fg_multi_solve(multi, cur.data(), &o, a.data(), b1.data(), b2.data(), flux.data(), info.data());
  fg_multi_timing t{};
  fg_multi_last_timing(multi, &t);
  *launches += static_cast<int>(t.pcg_launches);
  fg_multi_destroy(multi);
  for (size_t i = 0; i < M; ++i) {
    Solved &s = (*out)[where[i].first][where[i].second];
    *pcg_iterations += info[i].linear_iterations;
    s.iterations = info[i].iterations;
    s.residual = info[i].residual_l2;
    (*statuses)[where[i].first][where[i].second] = rc != 0 ? rc : info[i].status;
  }
  return true;
}

int SolveCurrents(Prepared &p, const std::vector<const std::vector<double> *> &currents, std::vector<Solved> *out,
                  std::vector<int> *statuses, int *launches)
{
  const fg_model m = p.artifact.Model();
  const size_t k = currents.size(), N = m.node_count, E = m.triangle_count, C = m.circuit_count;
  std::vector<double> cur(k * C), a(k * N), b1(k * E), b2(k * E), flux(k * (C ? C : 1));
  for (size_t i = 0; i < k; ++i)
    for (size_t c = 0; c < C; ++c)
      cur[i * C + c] = (*currents[i])[c];
  std::vector<fg_item_info> info(k);
  fg_solve_options o;
  fg_production_options(&o);
  const int rc = fg_solve_batch(p.plan, static_cast<int32_t>(k), cur.data(), nullptr, nullptr, &o, a.data(),
                                b1.data(), b2.data(), flux.data(), info.data());
  fg_timing t{};
  fg_plan_last_timing(p.plan, &t);
  *launches += static_cast<int>(t.pcg_launches);
  out->assign(k, Solved{});
  statuses->assign(k, rc);
  if (rc != 0)
    return rc;
  for (size_t i = 0; i < k; ++i) {
    Solved &s = (*out)[i];
    s.currents.assign(cur.begin() + i * C, cur.begin() + (i + 1) * C);
    s.flux.assign(flux.begin() + i * C, flux.begin() + i * C + C);
    s.a.assign(a.begin() + i * N, a.begin() + (i + 1) * N);
    s.b1.assign(b1.begin() + i * E, b1.begin() + (i + 1) * E);
    s.b2.assign(b2.begin() + i * E, b2.begin() + (i + 1) * E);
    s.iterations = info[i].iterations;
    s.residual = info[i].residual_l2;
    (*statuses)[i] = info[i].status;
  }
  return 0;
}

} // namespace fgcli
