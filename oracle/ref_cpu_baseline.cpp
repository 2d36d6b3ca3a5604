// ref_cpu_baseline.cpp -- the reference's CPU path for the timed CPU baseline.
//
// TEST/BENCHMARK INFRASTRUCTURE ONLY (compiled into oracle/_ref/libfemm_ref.so).
// One nonlinear solve is FEMM-GPU's host Newton assembler
// (AssembleNonlinearNewton + ReduceSignedSystem, gpu_solver/src/physics/
// nonlinear_model.cpp:453-627) feeding FEMM 4.2's own CPU sparse solver
// (CBigLinProb::PCGSolve, SSOR lambda = 1.5, fkn/spars.cpp:208-290), inside the
// Newton loop of NonlinearP1Solver::Solve (gpu_solver/src/solvers/
// nonlinear_solver.cu:667-769): cold secant at iteration 0, relaxation after
// iteration 5, the 1e-6 step gate and the adaptive inner tolerance.
//
// FEMM stops on the preconditioned residual sqrt(z'r / z0'b) < Precision; the
// GPU path stops on the true ||b - Ax|| / ||b||.  Each inner solve therefore
// starts with Precision = the Newton inner tolerance and tightens it tenfold
// (warm-restarting FEMM's PCG) until the true residual meets the same tolerance.
#include "physics/nonlinear_model.h"

#include "stdafx.h"
#include "fknDlg.h"
#include "complex.h"
#include "spars.h"

#include "femm_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <thread>
#include <vector>

using namespace gpu_femm;

extern "C" {
int ref_validate(const or_model *m);
}
bool RefModelFromOracle(const or_model *m, NonlinearModel *out); // ref_driver.cpp
int RefCpuNewtonModel(const NonlinearModel &model, int32_t k, const double *currents, const or_options *o,
                      int32_t threads, double *a_out, double *flux_out, int32_t *status,
                      int32_t *newton_iterations, int32_t *pcg_calls, double *max_true_residual);

namespace
{

bool BuildModel(const or_model *m, NonlinearModel *out) { return RefModelFromOracle(m, out); }

double TrueResidual(const Assembly &a, const std::vector<double> &rhs, const double *x)
{
  double num = 0.0, den = 0.0;
  for (size_t r = 0; r < rhs.size(); ++r) {
    double v = rhs[r];
    for (int k = a.row_offsets[r]; k < a.row_offsets[r + 1]; ++k)
      v -= a.values[k] * x[a.column_indices[k]];
    num += v * v;
    den += rhs[r] * rhs[r];
  }
  return den > 0.0 ? std::sqrt(num / den) : 0.0;
}

struct ItemResult {
  int status = 13;
  int newton_iterations = 0;
  int femm_pcg_calls = 0;
  double max_true_residual = 0.0;
};

// One sample's Newton solve as a state machine: Step() is one Newton iteration
// (host assembly + FEMM PCG to the inner tolerance + relaxation + step gate), so a
// benchmark can time a bounded number of iterations and resume the sample later.
class NewtonSample
{
public:
  NewtonSample(const NonlinearModel *model, NonlinearOptions options)
      : model_(model), options_(options)
  {
    const bool nonlinear = std::any_of(
        model->materials.begin(), model->materials.end(), [](const NonlinearMaterial &m) {
          return m.bh_curve_index >= 0 || m.alpha_per_t2 != 0.0;
        });
    options_.adaptive_linear_tolerance &= nonlinear;
  }

  void Start(const double *currents)
  {
    currents_.assign(currents, currents + model_->circuit_count);
    a_.assign(model_->nodes.size(), 0.0);
    for (size_t i = 0; i < model_->dirichlet_nodes.size(); ++i)
      a_[model_->dirichlet_nodes[i]] = model_->dirichlet_a_wb_per_m[i];
    relaxation_ = 1.0;
    previous_ = std::numeric_limits<double>::infinity();
    iteration_ = 0;
    done_ = false;
    result_ = ItemResult{};
    result_.status = static_cast<int>(Status::kNonlinearSolveNotConverged);
  }

  bool done() const { return done_; }
  const ItemResult &result() const { return result_; }
  const std::vector<double> &a() const { return a_; }

  // One Newton iteration; returns done().
  bool Step()
  {
    if (done_)
      return true;
    if (iteration_ >= options_.max_newton_iterations)
      return Finish(static_cast<int>(Status::kNonlinearSolveNotConverged));
    Assembly assembly;
    const Status status =
        AssembleNonlinearNewton(*model_, a_, currents_, iteration_ > 0, &assembly);
    if (status != Status::kOk)
      return Finish(static_cast<int>(status));
    const int n = static_cast<int>(assembly.free_nodes.size());
    std::vector<double> rhs(n);
    for (int r = 0; r < n; ++r)
      rhs[r] = assembly.rhs_per_amp[r] + assembly.rhs_offset[r];
    const double tolerance = NewtonLinearTolerance(options_, previous_);
    CFknDlg dialog;
    CBigLinProb linear;
    linear.Create(n, 0);
    linear.TheView = &dialog;
    for (int r = 0; r < n; ++r) {
      for (int k = assembly.row_offsets[r]; k < assembly.row_offsets[r + 1]; ++k)
        if (assembly.column_indices[k] >= r)
          linear.Put(assembly.values[k], r, assembly.column_indices[k]);
      linear.b[r] = rhs[r];
    }
    linear.Precision = tolerance;
    if (!linear.PCGSolve(0))
      return Finish(static_cast<int>(Status::kLinearSolveBreakdown));
    ++result_.femm_pcg_calls;
    double true_residual = TrueResidual(assembly, rhs, linear.V);
    while (true_residual > tolerance && linear.Precision > 1e-13) {
      linear.Precision *= 0.1;
      linear.PCGSolve(1);
      ++result_.femm_pcg_calls;
      true_residual = TrueResidual(assembly, rhs, linear.V);
    }
    result_.max_true_residual = std::max(result_.max_true_residual, true_residual);
    const std::vector<double> candidate =
        ExpandAssemblySolution(assembly, std::vector<double>(linear.V, linear.V + n));
    double difference_sq = 0.0, candidate_sq = 0.0;
    for (size_t i = 0; i < candidate.size(); ++i) {
      const double d = candidate[i] - a_[i];
      difference_sq += d * d;
      candidate_sq += candidate[i] * candidate[i];
    }
    const double residual = std::sqrt(difference_sq) /
                            std::max(std::sqrt(candidate_sq), std::numeric_limits<double>::min());
    if (!std::isfinite(residual))
      return Finish(static_cast<int>(Status::kNumericalNonfinite));
    if (iteration_ > 5) {
      if (residual > previous_ && relaxation_ > 0.125)
        relaxation_ *= 0.5;
      else
        relaxation_ += 0.1 * (1.0 - relaxation_);
    }
    for (size_t i = 0; i < a_.size(); ++i)
      a_[i] += relaxation_ * (candidate[i] - a_[i]);
    result_.newton_iterations = iteration_ + 1;
    if (NewtonStepConverged(options_, iteration_, residual, tolerance))
      return Finish(0);
    previous_ = residual;
    ++iteration_;
    return false;
  }

  // Flux linkage per circuit (nonlinear_solver.cu:36-42, :74-79, planar form).
  void Flux(double *flux_out) const
  {
    const NonlinearModel &model = *model_;
    for (int c = 0; c < model.circuit_count; ++c)
      flux_out[c] = 0.0;
    for (const NonlinearTriangle &t : model.triangles) {
      const NonlinearMaterial &mt = model.materials[t.material];
      if (mt.circuit_index < 0)
        continue;
      Node p[3] = {model.nodes[t.node[0]], model.nodes[t.node[1]], model.nodes[t.node[2]]};
      NonlinearElementTerms terms;
      BuildElementTerms(p, &terms);
      flux_out[mt.circuit_index] += terms.area_m2 * mt.source_j_per_a / 3.0 *
                                    (a_[t.node[0]] + a_[t.node[1]] + a_[t.node[2]]);
    }
    for (int c = 0; c < model.circuit_count; ++c)
      flux_out[c] *= model.depth_m;
  }

private:
  bool Finish(int status)
  {
    result_.status = status;
    done_ = true;
    return true;
  }

  const NonlinearModel *model_;
  NonlinearOptions options_;
  std::vector<double> currents_, a_;
  double relaxation_ = 1.0, previous_ = 0.0;
  int iteration_ = 0;
  bool done_ = false;
  ItemResult result_;
};

NonlinearOptions ToOptions(const or_options *o)
{
  NonlinearOptions options;
  options.relative_tolerance = o->relative_tolerance;
  options.max_newton_iterations = o->max_newton_iterations;
  options.max_linear_iterations = o->max_linear_iterations;
  options.linear_relative_tolerance = o->linear_relative_tolerance;
  options.recover_nonconvergence = o->recover_nonconvergence != 0;
  options.adaptive_linear_tolerance = o->adaptive_linear_tolerance != 0;
  return options;
}

// Runs fn(i) for i in [0, count) on `threads` host threads.
template <class F> void ParallelFor(int count, int threads, F fn)
{
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= count)
        return;
      fn(i);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < std::max(1, std::min(threads, count)); ++t)
    pool.emplace_back(worker);
  worker();
  for (auto &t : pool)
    t.join();
}

// A set of samples advanced one Newton iteration at a time (the bounded benchmark step).
struct Session {
  NonlinearModel model;
  std::vector<NewtonSample> samples;
};

} // namespace

extern "C" {

// Solves k independent samples of one planar model on `threads` host threads.
// currents [k*c]; a_out [k*N]; flux_out [k*c]; status/newton/pcg_calls [k];
// max_true_residual [k] = worst verified ||b-Ax||/||b|| of any inner solve.
int ref_cpu_newton_batch(const or_model *m, int32_t k, const double *currents,
                         const or_options *o, int32_t threads, double *a_out, double *flux_out,
                         int32_t *status, int32_t *newton_iterations, int32_t *pcg_calls,
                         double *max_true_residual)
{
  NonlinearModel model;
  if (m->problem_type != 0 || !BuildModel(m, &model))
    return static_cast<int>(Status::kInvalidArgument);
  return RefCpuNewtonModel(model, k, currents, o, threads, a_out, flux_out, status, newton_iterations,
                           pcg_calls, max_true_residual);
}
}

int RefCpuNewtonModel(const NonlinearModel &model, int32_t k, const double *currents, const or_options *o,
                      int32_t threads, double *a_out, double *flux_out, int32_t *status,
                      int32_t *newton_iterations, int32_t *pcg_calls, double *max_true_residual)
{
  const NonlinearOptions options = ToOptions(o);
  const size_t N = model.nodes.size();
  const int C = model.circuit_count;
  ParallelFor(k, threads, [&](int item) {
    NewtonSample sample(&model, options);
    sample.Start(currents + (size_t)item * C);
    while (!sample.Step()) {
    }
    std::copy(sample.a().begin(), sample.a().end(), a_out + (size_t)item * N);
    sample.Flux(flux_out + (size_t)item * C);
    const ItemResult &r = sample.result();
    status[item] = r.status;
    newton_iterations[item] = r.newton_iterations;
    pcg_calls[item] = r.femm_pcg_calls;
    max_true_residual[item] = r.max_true_residual;
  });
  return 0;
}

extern "C" {

// Session of k samples (currents [k*c]) for step-wise timing; *out receives the handle.
int ref_session_create(const or_model *m, int32_t k, const double *currents,
                       const or_options *o, void **out)
{
  *out = nullptr;
  auto *session = new Session;
  if (m->problem_type != 0 || !BuildModel(m, &session->model)) {
    delete session;
    return static_cast<int>(Status::kInvalidArgument);
  }
  const NonlinearOptions options = ToOptions(o);
  session->samples.reserve(k);
  for (int i = 0; i < k; ++i) {
    session->samples.emplace_back(&session->model, options);
    session->samples.back().Start(currents + (size_t)i * session->model.circuit_count);
  }
  *out = session;
  return 0;
}

// One Newton iteration of every unfinished sample, one sample per host thread.
// done [k] = 1 for samples that have finished (converged or failed).
int ref_session_step(void *handle, int32_t threads, int32_t *done)
{
  auto *session = static_cast<Session *>(handle);
  const int k = static_cast<int>(session->samples.size());
  ParallelFor(k, threads, [&](int i) { session->samples[i].Step(); });
  for (int i = 0; i < k; ++i)
    done[i] = session->samples[i].done() ? 1 : 0;
  return 0;
}

// Restarts sample i from the zero state with new currents [c].
int ref_session_restart(void *handle, int32_t i, const double *currents)
{
  auto *session = static_cast<Session *>(handle);
  if (i < 0 || i >= static_cast<int>(session->samples.size()))
    return static_cast<int>(Status::kInvalidArgument);
  session->samples[i].Start(currents);
  return 0;
}

// Per-sample status and Newton iterations so far.
int ref_session_info(void *handle, int32_t *status, int32_t *newton_iterations)
{
  auto *session = static_cast<Session *>(handle);
  for (size_t i = 0; i < session->samples.size(); ++i) {
    status[i] = session->samples[i].result().status;
    newton_iterations[i] = session->samples[i].result().newton_iterations;
  }
  return 0;
}

void ref_session_destroy(void *handle) { delete static_cast<Session *>(handle); }

} // extern "C"
