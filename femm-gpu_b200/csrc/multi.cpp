// multi.cpp -- heterogeneous batches (see multi.h).
#include "multi.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>

namespace fg
{
namespace
{

constexpr int kMinRowsPerCta = 1024; // below this a CTA's rows no longer pay for its barrier

} // namespace

Status MultiSolver::Create(std::vector<Plan *> plans, int kp)
{
  kp_ = kp;
  if (plans.empty())
    return Status::kInvalidArgument;
  for (Plan *p : plans)
    if (!p || p->host_only_ || p->options_.precision != FG_PRECISION_FP64 || p->block_size() != 0 ||
        p->from_iterate_ || p->one_reduction_)
      return p && p->host_only_ ? Status::kGpuUnavailable : Status::kUnsupportedFeature;
  for (size_t i = 0; i < plans.size(); ++i)
    for (size_t j = 0; j < i; ++j)
      if (plans[i] == plans[j])
        return Status::kInvalidArgument; // a plan's workspace serves one sample at a time
  plans_ = std::move(plans);
  max_grid_ = MultiPcgMaxGrid(kp_);
  if (max_grid_ <= 0)
    return kp_ == 1 || kp_ == kMaxItems ? Status::kGpuUnavailable : Status::kUnsupportedFeature;
  ring_ = MultiPcgRingBytes(kp_) > 0;
  const size_t m = plans_.size();
  Status s;
  if ((s = args_.ensure(m)) != Status::kOk || (s = cta_group_.ensure(max_grid_)) != Status::kOk ||
      (s = group_first_.ensure(m)) != Status::kOk || (s = group_size_.ensure(m)) != Status::kOk ||
      (s = host_args_.ensure(m)) != Status::kOk || (s = host_errors_.ensure(m)) != Status::kOk)
    return s;
  host_cta_group_.assign(max_grid_, 0);
  host_group_first_.assign(m, 0);
  host_group_size_.assign(m, 0);
  // Pinned copies of the maps so that a captured graph re-reads them on every replay.
  if ((s = pinned_maps_.ensure(static_cast<size_t>(max_grid_) + 2 * m)) != Status::kOk)
    return s;
  if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess)
    return Status::kInternalError;
  last_its_.assign(m, -1.0);
  return Status::kOk;
}

MultiSolver::~MultiSolver()
{
  if (graph_)
    cudaGraphExecDestroy(graph_);
  if (stream_)
    cudaStreamDestroy(stream_);
}

// The online tuner: every active plan gets one CTA, then the rest go, one at a time, to
// the plan with the largest predicted time per CTA, rows x iterations / CTAs, never more
// CTAs than rows / kMinRowsPerCta.  Returns the launch's CTA total (the same for a given
// active set, so a captured graph keeps its grid).
int MultiSolver::Partition(const std::vector<int> &active, std::vector<int> *ctas)
{
  const size_t a = active.size();
  ctas->assign(a, 1);
  std::vector<double> cost(a);
  std::vector<int> cap(a);
  int total_cap = 0;
  for (size_t i = 0; i < a; ++i) {
    const Plan &p = *plans_[active[i]];
    const double rows = p.host_.n;
    const double its = last_its_[active[i]] > 0 ? last_its_[active[i]] : sqrt_coeff_ * std::sqrt(rows);
    cost[i] = rows * its;
    cap[i] = std::max(1, static_cast<int>(rows / kMinRowsPerCta));
    total_cap += cap[i];
  }
  const int total = std::max(static_cast<int>(a), std::min(max_grid_, total_cap));
  int given = static_cast<int>(a);
  while (given < total) {
    int best = -1;
    double worst = -1.0;
    for (size_t i = 0; i < a; ++i)
      if ((*ctas)[i] < cap[i] && cost[i] / (*ctas)[i] > worst) {
        worst = cost[i] / (*ctas)[i];
        best = static_cast<int>(i);
      }
    if (best < 0)
      break;
    ++(*ctas)[best];
    ++given;
  }
  return given;
}

// One Newton step's device work for the active plans (captured or not): assembly, the
// multi-plan PCG, norms and the summaries to the host.
Status MultiSolver::Iteration(const std::vector<int> &active, cudaStream_t st)
{
  for (int m : active) {
    Plan &p = *plans_[m];
    Status s = p.ChunkAssemble(&chunks_[m]);
    if (s != Status::kOk)
      return s;
    if (cudaMemsetAsync(p.barrier_.get(), 0, sizeof(unsigned), st) != cudaSuccess ||
        cudaMemsetAsync(p.error_.get(), 0, sizeof(int32_t), st) != cudaSuccess)
      return Status::kInternalError;
  }
  const size_t a = active.size();
  const int32_t *maps = pinned_maps_.get();
  if (cudaMemcpyAsync(args_.get(), host_args_.get(), sizeof(PcgArgs) * a, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(cta_group_.get(), maps, sizeof(int32_t) * graph_ctas_, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(group_first_.get(), maps + max_grid_, sizeof(int32_t) * a, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(group_size_.get(), maps + max_grid_ + plans_.size(), sizeof(int32_t) * a,
                      cudaMemcpyHostToDevice, st) != cudaSuccess)
    return Status::kInternalError;
  PcgGroups g{args_.get(), cta_group_.get(), group_first_.get(), group_size_.get()};
  if (LaunchMultiPcg(g, kp_, graph_ctas_, st) != cudaSuccess)
    return Status::kInternalError;
  for (int m : active) {
    Status s = plans_[m]->ChunkNorms(&chunks_[m], true);
    if (s != Status::kOk)
      return s;
  }
  return Status::kOk;
}

// The lock-step Newton loop over the begun chunks_, then recovery and finish.
Status MultiSolver::Run(const fg_solve_options &options, std::vector<double> *first_its)
{
  const size_t M = plans_.size();
  for (;;) {
    std::vector<int> active;
    for (size_t m = 0; m < M; ++m)
      if (chunks_[m].valid && chunks_[m].active && chunks_[m].iteration < options.max_newton_iterations)
        active.push_back(static_cast<int>(m));
    if (active.empty())
      break;
    if (static_cast<int>(active.size()) > max_grid_)
      active.resize(max_grid_); // the rest wait for a later step (lock-step is not required)
    // Partition, tolerances and the PCG argument table (pinned; read by the graph).
    std::vector<int> ctas;
    const int total = Partition(active, &ctas);
    int32_t *maps = pinned_maps_.get();
    int next = 0;
    for (size_t i = 0; i < active.size(); ++i) {
      Plan &p = *plans_[active[i]];
      Plan::Chunk &c = chunks_[active[i]];
      p.ChunkTolerance(&c);
      if (c.kp != kp_ || !p.ChunkPcgArgs(c, p.barrier_.get(), p.error_.get(), host_args_.get() + i))
        return Status::kUnsupportedFeature;
      if (ring_) {
        host_args_.get()[i].value_ring = 1;
        host_args_.get()[i].value_ring_offset = 0;
      }
      maps[max_grid_ + i] = next;
      maps[max_grid_ + M + i] = ctas[i];
      for (int j = 0; j < ctas[i]; ++j)
        maps[next + j] = static_cast<int32_t>(i);
      next += ctas[i];
    }
    // A plan's first step assembles with the cold secant, later ones with the Jacobian:
    // only steps where no active plan is at its first iteration can replay a graph.
    bool first_step = false;
    for (int m : active)
      first_step = first_step || chunks_[m].iteration == 0;
    const bool reuse = graph_ && !first_step && active == graph_active_ && total == graph_ctas_;
    graph_ctas_ = total;
    timing_.max_ctas = std::max(timing_.max_ctas, total);
    Status s = Status::kOk;
    if (reuse) {
      if (cudaGraphLaunch(graph_, stream_) != cudaSuccess)
        return Status::kInternalError;
      ++timing_.graph_launches;
    } else if (!first_step && graphs_enabled_) {
      // Capture this step's sequence for the current active set, then replay it.
      if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
      }
      cudaGraph_t g = nullptr;
      bool ok = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        s = Iteration(active, stream_);
        ok = cudaStreamEndCapture(stream_, &g) == cudaSuccess && s == Status::kOk;
      }
      if (ok)
        ok = cudaGraphInstantiate(&graph_, g, 0) == cudaSuccess;
      if (g)
        cudaGraphDestroy(g);
      if (ok) {
        ++timing_.graph_captures;
        graph_active_ = active;
        if (cudaGraphLaunch(graph_, stream_) != cudaSuccess)
          return Status::kInternalError;
        ++timing_.graph_launches;
      } else {
        // Capture unsupported here: run this and every later step eagerly.
        cudaGetLastError();
        graph_ = nullptr;
        graphs_enabled_ = false;
        if ((s = Iteration(active, stream_)) != Status::kOk)
          return s;
      }
    } else {
      if ((s = Iteration(active, stream_)) != Status::kOk)
        return s;
    }
    ++timing_.pcg_launches;
    ++timing_.newton_steps;
    if (cudaStreamSynchronize(stream_) != cudaSuccess)
      return Status::kInternalError;
    for (int m : active) {
      Plan &p = *plans_[m];
      const double its = p.small_.get()[1]; // PCG iterations of item 0 this step
      if ((s = p.ChunkDecide(&chunks_[m])) != Status::kOk || (s = p.ChunkUpdate(&chunks_[m])) != Status::kOk)
        return s;
      last_its_[m] = std::max(1.0, its);
      if ((*first_its)[m] < 0)
        (*first_its)[m] = its;
    }
  }
  for (size_t m = 0; m < M; ++m) {
    if (!chunks_[m].valid)
      continue;
    Status s = plans_[m]->ChunkRecover(&chunks_[m]);
    if (s == Status::kOk)
      s = plans_[m]->ChunkFinish(&chunks_[m]);
    if (s != Status::kOk)
      return s;
  }
  if (cudaStreamSynchronize(stream_) != cudaSuccess)
    return Status::kInternalError;
  return Status::kOk;
}

Status MultiSolver::SolveChunks(const SolveRequest &req, const std::vector<int> &firsts,
                                const std::vector<int> &counts)
{
  const auto t0 = std::chrono::steady_clock::now();
  timing_ = fg_multi_timing{};
  const size_t M = plans_.size();
  if (firsts.size() != M || counts.size() != M || !req.info)
    return Status::kInvalidArgument;
  // The request's inputs were queued on its stream; the chunks run on stream_.
  if (cudaStreamSynchronize(req.stream) != cudaSuccess)
    return Status::kInternalError;
  reqs_.assign(M, req);
  chunks_.assign(M, Plan::Chunk{});
  std::vector<double> first_its(M, -1.0);
  for (size_t m = 0; m < M; ++m) {
    Plan &p = *plans_[m];
    reqs_[m].stream = stream_;
    p.timing_ = fg_timing{};
    chunks_[m].timed = false;
    const Status s = p.ChunkBegin(reqs_[m], firsts[m], counts[m], &chunks_[m], kp_);
    if (s != Status::kOk)
      return s;
    chunks_[m].timed = false;
  }
  const Status s = Run(req.options, &first_its);
  if (s != Status::kOk)
    return s;
  for (size_t m = 0; m < M; ++m)
    timing_.kernel_launches += plans_[m]->timing_.kernel_launches;
  timing_.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return Status::kOk;
}

Status MultiSolver::Solve(const double *const *currents, const fg_solve_options &options,
                          double *const *a_out, double *const *b1_out, double *const *b2_out,
                          double *const *flux_out, fg_item_info *info)
{
  const auto t0 = std::chrono::steady_clock::now();
  timing_ = fg_multi_timing{};
  const size_t M = plans_.size();
  if (!info)
    return Status::kInvalidArgument;
  reqs_.assign(M, SolveRequest{});
  chunks_.assign(M, Plan::Chunk{});
  std::vector<double> first_its(M, -1.0);
  for (size_t m = 0; m < M; ++m) {
    Plan &p = *plans_[m];
    const size_t N = p.host_.N, E = p.host_.E, C = p.host_.C;
    if ((C > 0 && (!currents || !currents[m])))
      return Status::kInvalidArgument;
    Status s;
    if ((C > 0 && (s = p.in_currents_.upload(currents[m], C)) != Status::kOk) ||
        (s = p.out_a_.ensure(N)) != Status::kOk || (s = p.out_b1_.ensure(E)) != Status::kOk ||
        (s = p.out_b2_.ensure(E)) != Status::kOk || (s = p.out_flux_.ensure(C > 0 ? C : 1)) != Status::kOk)
      return s;
    p.timing_ = fg_timing{};
  }
  // The uploads above ran on the legacy stream; the solve runs on stream_.
  if (cudaDeviceSynchronize() != cudaSuccess)
    return Status::kInternalError;
  for (size_t m = 0; m < M; ++m) {
    Plan &p = *plans_[m];
    Status s;
    SolveRequest &r = reqs_[m];
    r.items = 1;
    r.currents = p.in_currents_.get();
    r.options = options;
    r.a_out = p.out_a_.get();
    r.b1_out = p.out_b1_.get();
    r.b2_out = p.out_b2_.get();
    r.flux_out = p.out_flux_.get();
    r.info = info + m;
    r.stream = stream_;
    chunks_[m].timed = false;
    if ((s = p.ChunkBegin(r, 0, 1, &chunks_[m])) != Status::kOk)
      return s;
    chunks_[m].timed = false;
  }
  Status s0 = Run(options, &first_its);
  if (s0 != Status::kOk)
    return s0;
  for (size_t m = 0; m < M; ++m) {
    Plan &p = *plans_[m];
    const size_t N = p.host_.N, E = p.host_.E, C = p.host_.C;
    if ((a_out && a_out[m] && cudaMemcpy(a_out[m], p.out_a_.get(), N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (b1_out && b1_out[m] && cudaMemcpy(b1_out[m], p.out_b1_.get(), E * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (b2_out && b2_out[m] && cudaMemcpy(b2_out[m], p.out_b2_.get(), E * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (flux_out && flux_out[m] && C > 0 &&
         cudaMemcpy(flux_out[m], p.out_flux_.get(), C * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
      return Status::kInternalError;
    timing_.kernel_launches += p.timing_.kernel_launches;
  }
  // Refit the first-step iteration model: iterations ~ coeff * sqrt(rows).
  double num = 0.0;
  int cnt = 0;
  for (size_t m = 0; m < M; ++m)
    if (first_its[m] > 0) {
      num += first_its[m] / std::sqrt(static_cast<double>(plans_[m]->host_.n));
      ++cnt;
    }
  if (cnt)
    sqrt_coeff_ = num / cnt;
  timing_.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return Status::kOk;
}

} // namespace fg
