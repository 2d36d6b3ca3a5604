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

namespace
{

bool BuildModel(const or_model *m, NonlinearModel *out)
{
  NonlinearModel model;
  model.problem_type =
      m->problem_type == 1 ? MagneticProblemType::kAxisymmetric : MagneticProblemType::kPlanar;
  model.depth_m = m->depth_m;
  model.circuit_count = m->circuit_count;
  for (int i = 0; i < m->node_count; ++i)
    model.nodes.push_back({m->xy[2 * i], m->xy[2 * i + 1]});
  for (int c = 0; c < m->curve_count; ++c) {
    NonlinearBhCurve curve;
    for (int k = m->curve_offsets[c]; k < m->curve_offsets[c + 1]; ++k) {
      curve.b_t.push_back(m->curve_b[k]);
      curve.h_a_per_m.push_back(m->curve_h[k]);
    }
    if (!BuildNonlinearBhSpline(&curve))
      return false;
    model.bh_curves.push_back(curve);
  }
  for (int i = 0; i < m->mat_count; ++i) {
    NonlinearMaterial material;
    material.reluctivity_zero_m_per_h = m->nu0[i];
    material.alpha_per_t2 = m->alpha[i];
    material.source_j_per_a = m->j_per_a[i];
    material.h_c_a_per_m = m->hc[i];
    material.magnetization_deg = m->mag_deg[i];
    material.bh_curve_index = m->curve_index[i];
    material.circuit_index = m->circuit_index[i];
    model.materials.push_back(material);
  }
  for (int e = 0; e < m->tri_count; ++e)
    model.triangles.push_back({{m->tri[3 * e], m->tri[3 * e + 1], m->tri[3 * e + 2]}, m->tri_mat[e]});
  for (int i = 0; i < m->dir_count; ++i) {
    model.dirichlet_nodes.push_back(m->dir_nodes[i]);
    model.dirichlet_a_wb_per_m.push_back(m->dir_values[i]);
  }
  for (int i = 0; i < m->con_count; ++i) {
    SignedNodeConstraint constraint;
    constraint.node_a = m->con_a[i];
    constraint.node_b = m->con_b[i];
    constraint.sign = m->con_sign[i];
    model.node_constraints.push_back(constraint);
  }
  *out = std::move(model);
  return true;
}

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

ItemResult SolveOne(const NonlinearModel &model, const std::vector<double> &currents,
                    NonlinearOptions options, double *a_out, double *flux_out)
{
  ItemResult out;
  const bool nonlinear =
      std::any_of(model.materials.begin(), model.materials.end(), [](const NonlinearMaterial &m) {
        return m.bh_curve_index >= 0 || m.alpha_per_t2 != 0.0;
      });
  options.adaptive_linear_tolerance &= nonlinear;
  std::vector<double> a(model.nodes.size(), 0.0);
  for (size_t i = 0; i < model.dirichlet_nodes.size(); ++i)
    a[model.dirichlet_nodes[i]] = model.dirichlet_a_wb_per_m[i];
  double relaxation = 1.0, previous = std::numeric_limits<double>::infinity();
  CFknDlg dialog;
  out.status = static_cast<int>(Status::kNonlinearSolveNotConverged);
  for (int iteration = 0; iteration < options.max_newton_iterations; ++iteration) {
    Assembly assembly;
    const Status status = AssembleNonlinearNewton(model, a, currents, iteration > 0, &assembly);
    if (status != Status::kOk) {
      out.status = static_cast<int>(status);
      return out;
    }
    const int n = static_cast<int>(assembly.free_nodes.size());
    std::vector<double> rhs(n);
    for (int r = 0; r < n; ++r)
      rhs[r] = assembly.rhs_per_amp[r] + assembly.rhs_offset[r];
    const double tolerance = NewtonLinearTolerance(options, previous);
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
    if (!linear.PCGSolve(0)) {
      out.status = static_cast<int>(Status::kLinearSolveBreakdown);
      return out;
    }
    ++out.femm_pcg_calls;
    double true_residual = TrueResidual(assembly, rhs, linear.V);
    while (true_residual > tolerance && linear.Precision > 1e-13) {
      linear.Precision *= 0.1;
      linear.PCGSolve(1);
      ++out.femm_pcg_calls;
      true_residual = TrueResidual(assembly, rhs, linear.V);
    }
    out.max_true_residual = std::max(out.max_true_residual, true_residual);
    const std::vector<double> candidate =
        ExpandAssemblySolution(assembly, std::vector<double>(linear.V, linear.V + n));
    double difference_sq = 0.0, candidate_sq = 0.0;
    for (size_t i = 0; i < candidate.size(); ++i) {
      const double d = candidate[i] - a[i];
      difference_sq += d * d;
      candidate_sq += candidate[i] * candidate[i];
    }
    const double residual = std::sqrt(difference_sq) /
                            std::max(std::sqrt(candidate_sq), std::numeric_limits<double>::min());
    if (!std::isfinite(residual)) {
      out.status = static_cast<int>(Status::kNumericalNonfinite);
      return out;
    }
    if (iteration > 5) {
      if (residual > previous && relaxation > 0.125)
        relaxation *= 0.5;
      else
        relaxation += 0.1 * (1.0 - relaxation);
    }
    for (size_t i = 0; i < a.size(); ++i)
      a[i] += relaxation * (candidate[i] - a[i]);
    out.newton_iterations = iteration + 1;
    if (NewtonStepConverged(options, iteration, residual, tolerance)) {
      out.status = 0;
      break;
    }
    previous = residual;
  }
  std::copy(a.begin(), a.end(), a_out);
  // Flux linkage per circuit (nonlinear_solver.cu:36-42, :74-79, planar form).
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
                                  (a[t.node[0]] + a[t.node[1]] + a[t.node[2]]);
  }
  for (int c = 0; c < model.circuit_count; ++c)
    flux_out[c] *= model.depth_m;
  return out;
}

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
  NonlinearOptions options;
  options.relative_tolerance = o->relative_tolerance;
  options.max_newton_iterations = o->max_newton_iterations;
  options.max_linear_iterations = o->max_linear_iterations;
  options.linear_relative_tolerance = o->linear_relative_tolerance;
  options.recover_nonconvergence = o->recover_nonconvergence != 0;
  options.adaptive_linear_tolerance = o->adaptive_linear_tolerance != 0;
  const size_t N = model.nodes.size();
  const int C = model.circuit_count;
  std::atomic<int> next{0};
  auto worker = [&]() {
    for (;;) {
      const int item = next.fetch_add(1);
      if (item >= k)
        return;
      const std::vector<double> cur(currents + (size_t)item * C, currents + (size_t)(item + 1) * C);
      const ItemResult r = SolveOne(model, cur, options, a_out + (size_t)item * N,
                                    flux_out + (size_t)item * C);
      status[item] = r.status;
      newton_iterations[item] = r.newton_iterations;
      pcg_calls[item] = r.femm_pcg_calls;
      max_true_residual[item] = r.max_true_residual;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < std::max(1, threads); ++t)
    pool.emplace_back(worker);
  worker();
  for (auto &t : pool)
    t.join();
  return 0;
}

} // extern "C"
