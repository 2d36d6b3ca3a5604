// solver.h -- the plan object behind the C ABI: device-resident model, workspace and
// the batched Newton driver (the role of NonlinearP1Solver + DeviceNonlinearAssemblyPlan
// + GpuCsrSolver in gpu_solver/src/solvers/nonlinear_solver.cuh:32-85).
#pragma once

#include "femm_gpu.h"
#include "common.h"
#include "kernels.cuh"
#include "model.h"

#include <map>
#include <memory>
#include <vector>

namespace fg
{

class MultiSolver;

struct SolveRequest {
  int items = 0;
  const double *currents = nullptr; // device [items * C]
  const double *hc_scale = nullptr; // device [items] or null
  const double *warm = nullptr;     // device [items * N] or null
  fg_solve_options options{};
  double *a_out = nullptr, *b1_out = nullptr, *b2_out = nullptr, *flux_out = nullptr; // device
  fg_item_info *info = nullptr;                                                        // host
  cudaStream_t stream = nullptr;
  // Guarded warm start: an item starts from `warm` only if its equation residual there is
  // below the zero start's, otherwise from the zero start (fg_item_info.warm_start = 2).
  bool guard_warm = false;
};

class Plan
{
public:
  Plan() = default;
  Plan(const Plan &) = delete;
  Plan &operator=(const Plan &) = delete;
  ~Plan();
  Status Create(HostModel model, const fg_plan_options &options);
  // Gives a host-only plan its device side (upload, events); no-op on a device plan.
  Status AttachDevice();
  Status SolveDevice(const SolveRequest &request);
  // Host buffers in and out.  warm_device (device [items * N], used instead of the host
  // `warm`) and guard_warm serve the learned warm start.
  Status SolveHost(int items, const double *currents, const double *hc_scale, const double *warm,
                   const fg_solve_options &options, double *a_out, double *b1_out,
                   double *b2_out, double *flux_out, fg_item_info *info,
                   const double *warm_device = nullptr, bool guard_warm = false);
  Status Assemble(int items, const double *states, const double *currents,
                  const int32_t *use_newton, double *values, double *diagonal, double *rhs);
  Status PcgSolve(int items, const double *values, int values_per_item, const double *rhs,
                  double tolerance, int max_iterations, double *x, fg_linear_info *info);
  // SolveTangentMultiRhs: the consistent Newton Jacobian at base_a [N] and the circuit-
  // derivative solutions of `directions` [m][C] through one shared-operator PCG launch per
  // chunk; host arrays out (each may be NULL): da [m][N], db1 / db2 [m][E], dflux [m][C].
  Status SolveTangent(const double *base_a, const double *base_currents, int m, const double *directions,
                      const fg_solve_options &options, double *da, double *db1, double *db2,
                      double *dflux, fg_linear_info *info);

  const std::map<int, fg_pcg_shape> &pcg_shapes() const { return shapes_; }
  const HostPlan &host() const { return host_; }
  const HostModel &model() const { return model_; }
  const fg_timing &timing() const { return timing_; }
  size_t DeviceBytes() const;

private:
  Status DeviceInit();
  Status Upload();
  Status EnsureWorkspace(int kp);
  Status SolveChunk(const SolveRequest &request, int first, int count);
  // Shared-geometry batches wider than one launch: up to kMaxLanes chunks of 32 items, each
  // on its own lane workspace of this model (this plan is lane 0), advance together through
  // one multi-group PCG launch per Newton step (MultiSolver::SolveChunks).  FP64 Jacobi
  // from the zero or a plain warm start only; lanes are created on first use and kept.
  bool ChunksTogether(const SolveRequest &request) const;
  Status EnsureLanes(int lanes);
  Status SolveChunksTogether(const SolveRequest &request, int first, int chunks);
  std::vector<std::unique_ptr<Plan>> lanes_; // lanes 1 .. n (lane 0 is this plan)
  // The launch-shape autotuner (fg_plan_pcg_shapes): LaunchShaped launches a, after timing
  // the candidate shapes of a's key once (a short run of the same system) when unseen.
  cudaError_t LaunchShaped(PcgArgs a, int *grid, int *block, cudaStream_t stream);
  std::map<int, fg_pcg_shape> shapes_;
  std::unique_ptr<MultiSolver> lane_solver_;
  int lane_solver_lanes_ = 0;

public:
  // One chunk's Newton solve as steps, so that several plans can advance together
  // (MultiSolver): Begin, then per iteration Assemble, the linear solve (Linear, or the
  // shared multi-plan PCG), Norms, a stream synchronisation, Decide and Update; Finish.
  struct Chunk {
    const SolveRequest *req = nullptr;
    int first = 0, k = 0, kp = 0, iteration = 0;
    bool valid = false, adaptive = false, timed = true;
    uint32_t active = 0, warm_mask = 0, update = 0;
    const double *currents = nullptr, *hc = nullptr;
    double tol = 0.0;
    std::vector<double> relax, prev;
    double linfo[3 * kMaxItems];
    ItemScalars rel{};
  };
  // min_kp: the chunk's item slots are at least this many (a multi-group launch needs every
  // group at the same width).
  Status ChunkBegin(const SolveRequest &request, int first, int count, Chunk *c, int min_kp = 1);
  void ChunkTolerance(Chunk *c);
  Status ChunkAssemble(Chunk *c);
  Status ChunkLinear(Chunk *c);
  Status ChunkNorms(Chunk *c, bool linfo_on_device);
  Status ChunkDecide(Chunk *c);
  Status ChunkUpdate(Chunk *c);
  // SolveSafeguarded for the items the Newton loop exhausted (recover_nonconvergence).
  Status ChunkRecover(Chunk *c);
  Status ChunkFinish(Chunk *c);
  // The FP64 Jacobi PCG of this plan's current system for a multi-plan launch (barrier and
  // error flag supplied by the caller); false when the plan's options need another kernel.
  bool ChunkPcgArgs(const Chunk &c, unsigned *barrier, int32_t *error, PcgArgs *out);
  fg_timing &mutable_timing() { return timing_; }

private:
  friend class MultiSolver;
  Status RunPcg(int kp, int items, uint32_t mask, double tolerance, int max_iterations,
                int value_stride, int value_item, int diag_stride, int diag_item, int use_inverse,
                cudaStream_t stream, const double *blocks = nullptr, const double *b = nullptr,
                const double *item_tol = nullptr);
  // Block-Jacobi inverses of the current operators (values_, diag_) into blocks64_ or
  // blocks32_; no-op for the Jacobi preconditioner.
  Status BuildBlocks(int kp, int items, bool per_item, bool single, cudaStream_t stream);
  int block_size() const
  {
    return options_.preconditioner == FG_PRECOND_BLOCK_JACOBI ? options_.block_size : 0;
  }
  // The Newton linear solve of the active items: FP64 PCG, or FP32 PCG inside FP64 defect
  // correction.  linfo[3 * item] = status, iterations, residual; solution in x_.
  // final_tolerance: `tolerance` is the options' exact inner tolerance in the relaxed Newton
  // regime (steps that can converge after the first five), where the PCG from the iterate
  // solves tighter.
  Status LinearSolve(int kp, int items, uint32_t mask, double tolerance, int max_iterations,
                     cudaStream_t stream, double *linfo, bool final_tolerance = true);
  Status MixedSolve(int kp, int items, uint32_t mask, double tolerance, int max_iterations,
                    cudaStream_t stream, double *linfo, const double *b, const double *item_tol);

  HostModel model_;
  HostPlan host_;
  fg_plan_options options_{};
  DevicePlan dev_{};
  fg_timing timing_{};
  int kp_cap_ = 0;
  bool host_only_ = false;
  bool from_iterate_ = false; // FG_PLAN_PCG_FROM_ITERATE
  bool one_reduction_ = false; // FG_PLAN_PCG_ONE_REDUCTION
  int pcg_grid_cap_ = 0;
  int chunk_cap_ = kMaxItems; // items per batched launch

  // Plan constants on the device.
  DeviceArray<int32_t> row_offsets_, columns_, row_len_, slice_off_, sell_col_, contrib_off_,
      contrib_, rhs_off_, rhs_contrib_, elem_nodes_, elem_mat_, mat_curve_off_, mat_curve_cnt_,
      mat_circuit_, node_to_free_, free_roots_, circuit_elem_off_, circuit_elems_;
  DeviceArray<int8_t> node_sign_;
  DeviceArray<double> age_val_, age_rhs_; // allocated only with air-gap elements
  DeviceArray<double> pm_rhs_, circuit_rhs_, elem_geo_, mat_nu0_, mat_alpha_, mat_cold_, mat_jpa_,
      curve_b_, curve_h_, curve_slope_, boundary_;
  // Batch workspace.
  DeviceArray<double> state_, ev_, er_, values_, diag_, invd_, rhs_, x_, r_, z_, p0_, p1_, q_;
  DeviceArray<double> t0_, t1_; // the one-reduction form's extra vectors
  DeviceArray<double> norm_partials_, norms_, pcg_partials_, pcg_info_, staging_;
  // Mixed-precision form: FP32 operator, preconditioner and inner-solve vectors.
  DeviceArray<float> v32_, d32_, i32_, x32_, r32_, z32_, p032_, p132_, q32_;
  // Block-Jacobi inverses [n_pad * bs][KP] (FP64; FP32 for the mixed form's inner solve).
  DeviceArray<double> blocks64_;
  DeviceArray<float> blocks32_;
  DeviceArray<int32_t> block_fallbacks_;
  // PCG from the iterate: free-row state x0, defect d, per-item tolerances.
  DeviceArray<double> x0_, d_, item_tol_;
  DeviceArray<double> saved_; // recovery: the last accepted state [N][KP]
  Status EquationNorms(int kp, cudaStream_t st, double *res);
  DeviceArray<unsigned> barrier_;
  DeviceArray<unsigned long long> trace_;
  bool trace_enabled_ = false;
  DeviceArray<int32_t> error_, invalid_;
  // Host-pointer API staging.
  DeviceArray<double> in_currents_, in_hc_, in_warm_, out_a_, out_b1_, out_b2_, out_flux_;
  PinnedArray<double> small_;
  cudaEvent_t ev_start_ = nullptr, ev_mid_ = nullptr, ev_pcg_ = nullptr, ev_end_ = nullptr;
};

} // namespace fg

struct fg_plan {
  fg::Plan plan;
};
