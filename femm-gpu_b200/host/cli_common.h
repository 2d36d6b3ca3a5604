// cli_common.h -- pieces shared by the femm_gpu adapters: file I/O with atomic publication,
// prepared (read, verified, parsed, planned) artifacts, solved samples and their
// postprocess.
#pragma once

#include "artifact.h"
#include "femm_gpu.h"

#include <cstdint>
#include <map>
#include <memory>
#include <ostream>
#include <string>
#include <utility>
#include <vector>

namespace fgcli
{

constexpr double kTwoPi = 6.283185307179586476925286766559005768;
constexpr double kPi = 3.141592653589793238462643383279502884;

struct Options {
  fg_plan_options plan{FG_PRECOND_JACOBI, 8, FG_PRECISION_FP64, 0};
};

std::string StatusName(int s);
bool ReadFile(const std::string &path, std::string *out);
// Same file (by device and inode when both exist, else by resolved path).
bool SameFile(const std::string &a, const std::string &b);
// Writes `text` to path.tmp.<clock>.<n> and renames it over `path`.
bool PublishAtomically(const std::string &path, const std::string &text);

// What one solved sample returns.
struct Solved {
  std::vector<double> currents, flux, a, b1, b2;
  int32_t iterations = 0;
  double residual = 0.0;
};

// A postprocessed sample.
struct Post {
  double fx = 0.0, fy = 0.0, torque = 0.0;
  std::vector<double> radial;
};

template <class V> void List(std::ostream &o, const V &v)
{
  for (size_t i = 0; i < v.size(); ++i)
    o << (i ? ", " : "") << v[i];
}

fg_postprocess_options PostOptions(int32_t selected_group, int32_t air_group, double radius_mm,
                                   const std::vector<double> &angles_deg, std::vector<double> *angles);
// Postprocesses one solved sample on `pp` (created for the same request options).
int RunPost(fg_postprocess *pp, const Solved &s, Post *out);

// Postprocess objects of one artifact's plan, one per distinct request (groups, circle).
class PostCache
{
public:
  ~PostCache()
  {
    for (auto &kv : cache_)
      if (kv.second.second)
        fg_postprocess_destroy(kv.second.second);
  }
  // Status of the postprocess plan of (selected group, air group, circle); *pp valid when 0.
  // angles_rad replaces the converted angles (sector probes folded into the representative
  // sector); apex lists the symmetry apex nodes the mask does not fix.
  int Get(fg_plan *plan, int32_t selected_group, int32_t air_group, double radius_mm,
          const std::vector<double> &angles_deg, fg_postprocess **pp,
          const std::vector<double> *angles_rad = nullptr, const std::vector<int32_t> *apex = nullptr)
  {
    std::vector<double> key{static_cast<double>(selected_group), static_cast<double>(air_group), radius_mm,
                            angles_rad ? 1.0 : 0.0};
    key.insert(key.end(), angles_deg.begin(), angles_deg.end());
    auto it = cache_.find(key);
    if (it == cache_.end()) {
      std::vector<double> angles;
      fg_postprocess_options o = PostOptions(selected_group, air_group, radius_mm, angles_deg, &angles);
      if (angles_rad) {
        angles = *angles_rad;
        o.airgap_angles_rad = angles.data();
        o.airgap_angle_count = static_cast<int32_t>(angles.size());
      }
      if (apex && !apex->empty()) {
        o.symmetry_apex_count = static_cast<int32_t>(apex->size());
        o.symmetry_apex_nodes = apex->data();
      }
      fg_postprocess *p = nullptr;
      const int rc = fg_postprocess_create(plan, &o, nullptr, &p);
      it = cache_.emplace(key, std::make_pair(rc, p)).first;
    }
    *pp = it->second.second;
    return it->second.first;
  }

private:
  std::map<std::vector<double>, std::pair<int, fg_postprocess *>> cache_;
};

// A verified, parsed artifact and its plan.
struct Prepared {
  int status = 0;
  std::string error;
  fgio::Artifact artifact;
  fg_plan *plan = nullptr;
  int plan_status = -1;   // -1 not attempted, else the fg_plan_create status
  bool host_only = false; // a host-only plan still to be given its device side
  PostCache post;         // postprocess masks of this artifact, per request options
  // A v3 sector's tangent operator: the same mesh with the suspension order's boundary
  // relation (MakeMotorSectorTangentModel), built on first use.
  std::shared_ptr<Prepared> sector_tangent;
  bool sector_tangent_tried = false;
  // A sliding-band artifact's poses: per requested rotor angle a copy of the artifact with
  // its bands slid to that angle, and that copy's own plan (the operator differs per angle).
  std::map<double, std::shared_ptr<Prepared>> poses;
  uint64_t pose_clock = 0, last_use = 0; // pose recency (PoseOf), for TrimPoses
  ~Prepared()
  {
    if (plan)
      fg_plan_destroy(plan);
  }
};

// Reads the artifact, checks its SHA-256 and parses it (the adapters' artifact gate).
void Prepare(const std::string &path, const std::string &sha, const Options &opt, Prepared *p);
// Builds the host side of the plan ahead of the GPU work (the streaming worker's prefetch).
void PreparePlanOnHost(Prepared *p, const Options &opt);
// The plan (NonlinearP1Solver::Initialize), created once the requests have matched.
int EnsurePlan(Prepared *p, const Options &opt);

// The Prepared that solves rotor_angle_deg: `p` itself for a conforming artifact, else its
// sliding-band pose at that angle, made on first use (ApplySlidingBandRotorAngle,
// sample_request.cpp:493-497; status FG_INVALID_ARGUMENT when the angle cannot be applied).
Prepared *PoseOf(Prepared &p, double rotor_angle_deg);
// Keeps the `keep` most recently used poses of a sliding-band artifact and frees the
// others' plans; call between chunks, when no pose is in use (a long-running worker meets
// ever new rotor angles).
void TrimPoses(Prepared &p, size_t keep);
constexpr size_t kResidentPoses = 64;
// The sliding-band postprocess of one solved sample (ComputeAirGapElementPostprocess via
// fg_air_gap_postprocess) at the request's probe angles in degrees.
// angles_rad, when given, replaces the converted angles (native sector probes folded into
// the representative sector).
int AirGapPost(fg_plan *plan, const Solved &s, const std::vector<double> &angles_deg, Post *out,
               const std::vector<double> *angles_rad = nullptr);

// One operator of a multi-operator solve: a prepared plan (an artifact, or a sliding-band
// pose) and the circuit currents of its samples.
struct Operator {
  Prepared *p = nullptr;
  std::vector<const std::vector<double> *> currents;
};
constexpr size_t kMultiGroupItems = 8;
// The samples of several operators in one multi-plan launch per Newton step (fg_multi).
// At motor mesh sizes each operator's own PCG launch is latency-bound, so solving them side
// by side amortises every CG iteration's barriers over all of them.  An operator's first
// sample runs on its plan, further samples on replica plans of the same model (the
// multi-plan launch takes one sample per plan; the replicas are freed when the solve
// ends).  Only the plain FP64 Jacobi form (the
// multi-plan kernel's), at least two operators and at most kMultiGroupItems samples per
// operator (a large group is better served by its own batched launch); otherwise false and
// nothing is solved.  out[o][j] / statuses[o][j]: sample j of operator o.
bool SolveOperatorsTogether(const std::vector<Operator> &ops, const Options &opt,
                            std::vector<std::vector<Solved>> *out, std::vector<std::vector<int>> *statuses,
                            int *launches, int64_t *pcg_iterations);

// Solves k samples (their circuit currents) on a prepared plan with the reference's
// production options (ProductionSampleOptions); statuses[i] = the item's status.
int SolveCurrents(Prepared &p, const std::vector<const std::vector<double> *> &currents, std::vector<Solved> *out,
                  std::vector<int> *statuses, int *launches);

using ArtifactKey = std::pair<std::string, std::string>; // path, SHA-256
using ArtifactCache = std::map<ArtifactKey, std::shared_ptr<Prepared>>;

} // namespace fgcli
