// multi.h -- heterogeneous batches: independent meshes (one plan each) solved together.
#pragma once

#include "solver.h"

#include <vector>

namespace fg
{

// Newton solves of one sample on each of several plans (meshes of any size), advanced in
// lock-step: per Newton iteration the assemblies of all active plans, ONE cooperative PCG
// launch in which every plan's solve runs on its own group of CTAs (MultiPcgKernel), and
// the norms.  From the second iteration on, that sequence is captured once per set of
// active plans into a CUDA graph and replayed (the PCG tolerances travel in a pinned table
// the graph copies to the device on every replay).  The CTAs of the launch are divided by
// an online tuner: a plan's share follows its predicted cost, rows x iterations, with the
// iterations of its previous Newton step (the first step uses c sqrt(rows), c fitted to
// the plans already solved by this object).
class MultiSolver
{
public:
  MultiSolver() = default;
  MultiSolver(const MultiSolver &) = delete;
  MultiSolver &operator=(const MultiSolver &) = delete;
  ~MultiSolver();
  // kp: items per group of the launch (1: one sample per plan; 32: chunks of a wide batch).
  Status Create(std::vector<Plan *> plans, int kp = 1);
  Status Solve(const double *const *currents, const fg_solve_options &options, double *const *a_out,
               double *const *b1_out, double *const *b2_out, double *const *flux_out, fg_item_info *info);
  // Chunks of one shared-geometry request: plan m (a lane workspace of the request's model,
  // created with kp = 32) solves items [firsts[m], firsts[m] + counts[m]) of req, writing
  // req's device outputs and host item infos.  The request's stream is not used: the solve
  // runs on this object's stream, ordered after everything queued before the call.
  Status SolveChunks(const SolveRequest &req, const std::vector<int> &firsts, const std::vector<int> &counts);
  const fg_multi_timing &timing() const { return timing_; }

private:
  // CTA counts for the active plans; returns the launch's CTA total.
  int Partition(const std::vector<int> &active, std::vector<int> *ctas);
  Status Iteration(const std::vector<int> &active, cudaStream_t st);
  // The lock-step Newton loop over chunks_ (begun) and its recovery and finish.
  Status Run(const fg_solve_options &options, std::vector<double> *first_its);

  std::vector<Plan *> plans_;
  std::vector<SolveRequest> reqs_;
  std::vector<Plan::Chunk> chunks_;
  std::vector<double> last_its_;   // PCG iterations of each plan's previous Newton step
  double sqrt_coeff_ = 4.0;        // fitted: iterations ~ coeff * sqrt(rows)
  int max_grid_ = 0;
  int kp_ = 1;
  bool ring_ = false; // the launch carries the value ring (dynamic shared memory)
  DeviceArray<PcgArgs> args_;
  DeviceArray<int32_t> cta_group_, group_first_, group_size_;
  DeviceArray<unsigned> barriers_;
  DeviceArray<int32_t> errors_;
  PinnedArray<PcgArgs> host_args_;
  PinnedArray<int32_t> host_errors_;
  PinnedArray<int32_t> pinned_maps_; // [max_grid] CTA -> group, [M] first CTA, [M] CTA count
  bool graphs_enabled_ = true;
  std::vector<int32_t> host_cta_group_, host_group_first_, host_group_size_;
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  std::vector<int> graph_active_;
  int graph_ctas_ = 0;
  fg_multi_timing timing_{};
};

} // namespace fg

struct fg_multi {
  fg::MultiSolver solver;
};
