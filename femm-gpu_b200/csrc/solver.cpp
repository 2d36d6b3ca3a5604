// solver.cpp -- batched Newton driver over the device plan.
//
// Newton semantics follow NonlinearP1Solver::SolveBatch (gpu_solver/src/solvers/
// nonlinear_solver.cu:183-530) with the device-assembly path: zero start with the
// expanded fixed values, cold-secant operator at iteration zero (Newton from the
// start for a warm-started item, as Solve() does at :698), one inner tolerance for
// the batch = the tightest NewtonLinearTolerance of its active items
// (nonlinear_model.cpp:166-184), relaxation after iteration five, the 1e-6 step gate
// at the exact inner tolerance (NewtonStepConverged, :186-193), per-item status
// isolation.  Everything stays on the device except 2 x items step norms and the PCG
// summaries that cross back once per Newton iteration.
#include "solver.h"

#include "multi.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <limits>

namespace fg
{
namespace
{

int PadItems(int k)
{
  int kp = 1;
  while (kp < k)
    kp <<= 1;
  return kp;
}

double NewtonLinearTolerance(const fg_solve_options &o, bool adaptive, double previous_step)
{
  const double exact = o.linear_relative_tolerance;
  if (!adaptive || !std::isfinite(previous_step) || previous_step <= 100.0 * o.relative_tolerance ||
      !(exact > 0.0) || !std::isfinite(exact))
    return exact;
  return std::max(exact, 1e-8 * std::min(1.0, previous_step));
}

float Elapsed(cudaEvent_t a, cudaEvent_t b)
{
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.0f;
  }
  return ms;
}

// Chunks of a wide shared-geometry batch solved together in one multi-group launch.
constexpr int kMaxLanes = 32;

// The PCG from the iterate at the exact inner tolerance, in the relaxed Newton regime,
// solves to this fraction of it, but not below kIterateFinalFloor (nor below a tolerance
// the caller set tighter still): the FP64 true residual of a 1e-14 target is not reliably
// reachable.
constexpr double kIterateFinalTightening = 0.1;
constexpr double kIterateFinalFloor = 1e-12;

// FG_CHUNKS_TOGETHER in the environment (read at every solve): unset or 0 solves wide
// batches chunk after chunk (the default: measured faster on the B200 from 1.5k to 40k
// rows); 1 advances the chunks together where the L2 rule of Plan::SolveDevice allows, 2
// whatever their footprint.
int ChunksTogetherMode()
{
  const char *v = std::getenv("FG_CHUNKS_TOGETHER");
  return v && v[0] == '1' ? 1 : (v && v[0] == '2' ? 2 : 0);
}

// Bytes of the vectors one chunk of kMaxItems items keeps in use per CG iteration (x, r,
// z, two directions, q, b, the diagonal and its inverse; FP64), which the PCG needs resident
// in L2 to run at speed.
size_t ChunkVectorBytes(int64_t n_pad) { return static_cast<size_t>(n_pad) * kMaxItems * 8 * 9; }

} // namespace

Plan::~Plan()
{
  lane_solver_.reset();
  lanes_.clear();
  for (cudaEvent_t e : {ev_start_, ev_mid_, ev_pcg_, ev_end_})
    if (e)
      cudaEventDestroy(e);
}

size_t Plan::DeviceBytes() const
{
  size_t b = 0;
  b += row_offsets_.bytes() + columns_.bytes() + row_len_.bytes() + slice_off_.bytes() +
       sell_col_.bytes() + contrib_off_.bytes() + contrib_.bytes() + rhs_off_.bytes() +
       rhs_contrib_.bytes() + elem_nodes_.bytes() + elem_mat_.bytes() + node_to_free_.bytes() +
       free_roots_.bytes() +
       circuit_elem_off_.bytes() + circuit_elems_.bytes() + node_sign_.bytes() + pm_rhs_.bytes() +
       circuit_rhs_.bytes() + elem_geo_.bytes() + boundary_.bytes();
  b += state_.bytes() + ev_.bytes() + er_.bytes() + values_.bytes() + diag_.bytes() +
       invd_.bytes() + rhs_.bytes() + x_.bytes() + r_.bytes() + z_.bytes() + p0_.bytes() +
       p1_.bytes() + q_.bytes() + t0_.bytes() + t1_.bytes() + pcg_partials_.bytes() + staging_.bytes();
  b += in_currents_.bytes() + in_hc_.bytes() + in_warm_.bytes() + out_a_.bytes() + out_b1_.bytes() +
       out_b2_.bytes() + out_flux_.bytes();
  return b;
}

Status Plan::Create(HostModel model, const fg_plan_options &options)
{
  model_ = std::move(model);
  options_ = options;
  if ((options_.preconditioner != FG_PRECOND_JACOBI &&
       options_.preconditioner != FG_PRECOND_BLOCK_JACOBI) ||
      (options_.preconditioner == FG_PRECOND_BLOCK_JACOBI && options_.block_size != 8 &&
       options_.block_size != 32) ||
      (options_.precision != FG_PRECISION_FP64 && options_.precision != FG_PRECISION_MIXED))
    return Status::kUnsupportedFeature;
  // 32-row blocks in FP64 (the mixed form's fallback included) stop at 16 items per launch.
  chunk_cap_ = block_size() == 32 ? 16 : kMaxItems;
  Status s = BuildHostPlan(model_, &host_);
  if (s != Status::kOk)
    return s;
  if (host_.E >= (1 << 27) || host_.positions > (int64_t(1) << 31) / kMaxItems)
    return Status::kUnsupportedFeature;
  host_only_ = (options_.flags & FG_PLAN_HOST_ONLY) != 0;
  from_iterate_ = (options_.flags & FG_PLAN_PCG_FROM_ITERATE) != 0;
  one_reduction_ = (options_.flags & FG_PLAN_PCG_ONE_REDUCTION) != 0;
  if (one_reduction_ && (options_.precision != FG_PRECISION_FP64 || block_size() != 0))
    return Status::kUnsupportedFeature;
  if (host_only_)
    return Status::kOk;
  return DeviceInit();
}

Status Plan::AttachDevice()
{
  if (!host_only_)
    return Status::kOk;
  const Status s = DeviceInit();
  if (s == Status::kOk) {
    host_only_ = false;
    options_.flags &= ~FG_PLAN_HOST_ONLY;
  }
  return s;
}

Status Plan::DeviceInit()
{
  Status s = Status::kOk;
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices < 1) {
    cudaGetLastError();
    return Status::kGpuUnavailable;
  }
  s = Upload();
  if (s != Status::kOk)
    return s;
  const char *trace = std::getenv("FG_PCG_TRACE");
  trace_enabled_ = trace && trace[0] == '1';
  if (trace_enabled_ && (s = trace_.ensure(kPcgTraceSlots)) != Status::kOk)
    return s;
  if (cudaEventCreate(&ev_start_) != cudaSuccess || cudaEventCreate(&ev_mid_) != cudaSuccess ||
      cudaEventCreate(&ev_pcg_) != cudaSuccess || cudaEventCreate(&ev_end_) != cudaSuccess)
    return Status::kInternalError;
  return Status::kOk;
}

Status Plan::Upload()
{
  const HostPlan &h = host_;
  Status s = Status::kOk;
#define FG_UP(dst, vec)                                                                            \
  if (s == Status::kOk)                                                                            \
    s = dst.upload(vec.data(), vec.size());
  FG_UP(row_offsets_, h.row_offsets);
  FG_UP(columns_, h.columns);
  FG_UP(row_len_, h.row_len);
  FG_UP(slice_off_, h.slice_off);
  FG_UP(sell_col_, h.sell_col);
  FG_UP(contrib_off_, h.contrib_off);
  FG_UP(contrib_, h.contrib);
  FG_UP(rhs_off_, h.rhs_off);
  FG_UP(rhs_contrib_, h.rhs_contrib);
  FG_UP(elem_nodes_, h.elem_nodes);
  FG_UP(elem_mat_, h.elem_mat);
  FG_UP(mat_curve_off_, h.mat_curve_off);
  FG_UP(mat_curve_cnt_, h.mat_curve_cnt);
  FG_UP(mat_circuit_, h.mat_circuit);
  FG_UP(node_to_free_, h.dofs.node_to_free);
  FG_UP(free_roots_, h.dofs.free_roots);
  FG_UP(circuit_elem_off_, h.circuit_elem_off);
  FG_UP(circuit_elems_, h.circuit_elems);
  FG_UP(node_sign_, h.dofs.node_sign);
  FG_UP(pm_rhs_, h.pm_rhs);
  FG_UP(circuit_rhs_, h.circuit_rhs);
  FG_UP(elem_geo_, h.elem_geo);
  FG_UP(mat_nu0_, h.mat_nu0);
  FG_UP(mat_alpha_, h.mat_alpha);
  FG_UP(mat_cold_, h.mat_cold);
  FG_UP(mat_jpa_, h.mat_jpa);
  FG_UP(curve_b_, h.curve_b);
  FG_UP(curve_h_, h.curve_h);
  FG_UP(curve_slope_, h.curve_slope);
  FG_UP(boundary_, h.dofs.boundary);
  if (!h.age_val.empty()) {
    FG_UP(age_val_, h.age_val);
    FG_UP(age_rhs_, h.age_rhs);
  }
#undef FG_UP
  if (s != Status::kOk)
    return s;
  if (cudaDeviceSynchronize() != cudaSuccess)
    return Status::kInternalError;
  DevicePlan &d = dev_;
  d.N = h.N;
  d.E = h.E;
  d.n = h.n;
  d.n_pad = h.n_pad;
  d.slices = h.slices;
  d.C = h.C;
  d.problem_type = h.problem_type;
  d.nnz = h.nnz;
  d.positions = h.positions;
  d.row_offsets = row_offsets_.get();
  d.columns = columns_.get();
  d.row_len = row_len_.get();
  d.slice_off = slice_off_.get();
  d.sell_col = sell_col_.get();
  d.contrib_off = contrib_off_.get();
  d.contrib = contrib_.get();
  d.rhs_off = rhs_off_.get();
  d.rhs_contrib = rhs_contrib_.get();
  d.pm_rhs = pm_rhs_.get();
  d.circuit_rhs = circuit_rhs_.get();
  d.age_val = h.age_val.empty() ? nullptr : age_val_.get();
  d.age_rhs = h.age_val.empty() ? nullptr : age_rhs_.get();
  d.elem_nodes = elem_nodes_.get();
  d.elem_mat = elem_mat_.get();
  d.elem_geo = elem_geo_.get();
  d.mat_nu0 = mat_nu0_.get();
  d.mat_alpha = mat_alpha_.get();
  d.mat_cold = mat_cold_.get();
  d.mat_jpa = mat_jpa_.get();
  d.mat_curve_off = mat_curve_off_.get();
  d.mat_curve_cnt = mat_curve_cnt_.get();
  d.mat_circuit = mat_circuit_.get();
  d.curve_b = curve_b_.get();
  d.curve_h = curve_h_.get();
  d.curve_slope = curve_slope_.get();
  d.node_to_free = node_to_free_.get();
  d.free_roots = free_roots_.get();
  d.node_sign = node_sign_.get();
  d.boundary = boundary_.get();
  d.circuit_elem_off = circuit_elem_off_.get();
  d.circuit_elems = circuit_elems_.get();
  d.depth_m = model_.depth_m;
  return Status::kOk;
}

Status Plan::EnsureWorkspace(int kp)
{
  if (kp <= kp_cap_)
    return Status::kOk;
  const HostPlan &h = host_;
  const size_t vec = static_cast<size_t>(h.n_pad) * kp;
  Status s = Status::kOk;
  const int grid = PcgMaxGrid(kp);
  if (grid <= 0)
    return Status::kGpuUnavailable;
  pcg_grid_cap_ = std::max(pcg_grid_cap_, grid);
#define FG_EN(arr, count)                                                                          \
  if (s == Status::kOk)                                                                            \
    s = arr.ensure(count);
  FG_EN(state_, static_cast<size_t>(h.N) * kp);
  FG_EN(ev_, static_cast<size_t>(6) * h.E * kp);
  FG_EN(er_, static_cast<size_t>(3) * h.E * kp);
  FG_EN(values_, static_cast<size_t>(h.positions) * kp);
  FG_EN(diag_, vec);
  FG_EN(invd_, vec);
  FG_EN(rhs_, vec);
  FG_EN(x_, vec);
  FG_EN(r_, vec);
  FG_EN(z_, vec);
  FG_EN(p0_, vec);
  FG_EN(p1_, vec);
  FG_EN(q_, vec);
  FG_EN(norm_partials_, static_cast<size_t>(2) * kp * 256);
  FG_EN(norms_, static_cast<size_t>(2) * kp);
  FG_EN(pcg_partials_, PcgPartialsDoubles(pcg_grid_cap_, one_reduction_));
  if (one_reduction_) {
    FG_EN(t0_, vec);
    FG_EN(t1_, vec);
  }
  FG_EN(pcg_info_, static_cast<size_t>(3) * kp);
  FG_EN(barrier_, 1);
  FG_EN(error_, 1);
  FG_EN(invalid_, static_cast<size_t>(kp));
  FG_EN(small_, static_cast<size_t>(10) * kp + 8); // summary [0, 7kp), recovery [7kp, 10kp)
  FG_EN(x0_, vec);
  FG_EN(saved_, static_cast<size_t>(h.N) * kp);
  FG_EN(d_, vec);
  FG_EN(item_tol_, static_cast<size_t>(kp));
  if (block_size() > 0) {
    FG_EN(blocks64_, vec * block_size());
    FG_EN(block_fallbacks_, 1);
    if (options_.precision == FG_PRECISION_MIXED)
      FG_EN(blocks32_, vec * block_size());
  }
  if (options_.precision == FG_PRECISION_MIXED) {
    FG_EN(v32_, static_cast<size_t>(h.positions) * kp);
    FG_EN(d32_, vec);
    FG_EN(i32_, vec);
    FG_EN(x32_, vec);
    FG_EN(r32_, vec);
    FG_EN(z32_, vec);
    FG_EN(p032_, vec);
    FG_EN(p132_, vec);
    FG_EN(q32_, vec);
  }
#undef FG_EN
  if (s != Status::kOk)
    return s;
  if (block_fallbacks_.get() && cudaMemset(block_fallbacks_.get(), 0, sizeof(int32_t)) != cudaSuccess)
    return Status::kInternalError;
  kp_cap_ = kp;
  return Status::kOk;
}

Status Plan::RunPcg(int kp, int items, uint32_t mask, double tolerance, int max_iterations,
                    int value_stride, int value_item, int diag_stride, int diag_item,
                    int use_inverse, cudaStream_t stream, const double *blocks, const double *b,
                    const double *item_tol)
{
  PcgArgs a{};
  a.item_tolerance = item_tol;
  if (blocks) {
    a.blocks = blocks;
    a.block_size = block_size();
    a.block_stride = value_stride;
    a.block_item = value_item;
  }
  a.n = host_.n;
  a.n_pad = host_.n_pad;
  a.slices = host_.slices;
  a.kp = kp;
  a.items = items;
  a.slice_off = slice_off_.get();
  a.host_slice_off = host_.slice_off.data();
  a.row_len = row_len_.get();
  a.sell_col = sell_col_.get();
  a.values = values_.get();
  a.value_stride = value_stride;
  a.value_item = value_item;
  a.diag = diag_.get();
  a.invd = invd_.get();
  a.diag_stride = diag_stride;
  a.diag_item = diag_item;
  a.use_inverse = use_inverse;
  a.b = b ? b : rhs_.get();
  a.x = x_.get();
  a.r = r_.get();
  a.z = z_.get();
  a.p0 = p0_.get();
  a.p1 = p1_.get();
  a.q = q_.get();
  if (one_reduction_ && !blocks) {
    a.one_reduction = 1;
    a.t0 = t0_.get();
    a.t1 = t1_.get();
  }
  a.partials = pcg_partials_.get();
  a.barrier = barrier_.get();
  a.error = error_.get();
  a.info = pcg_info_.get();
  a.tolerance = tolerance;
  a.max_iterations = max_iterations;
  a.active_mask = mask;
  a.timeout_ns = PcgWaitLimitNs();
  a.trace = trace_enabled_ ? trace_.get() : nullptr;
  int grid = 0, block = 0;
  const cudaError_t e = LaunchShaped(a, &grid, &block, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return Status::kInternalError;
  }
  timing_.pcg_grid = grid;
  timing_.pcg_block = block;
  timing_.pcg_launches += 1;
  timing_.kernel_launches += 1;
  return Status::kOk;
}

namespace
{
// CG iterations of each timed candidate launch, and rounds over the candidates.
constexpr int kTuneIterations = 64;
constexpr int kTuneRounds = 2;

bool TuningEnabled()
{
  const char *v = std::getenv("FG_PCG_TUNE");
  return !(v && v[0] == '0');
}
} // namespace

cudaError_t Plan::LaunchShaped(PcgArgs a, int *grid, int *block, cudaStream_t stream)
{
  const int key = a.kp * 1000 + a.precision * 100 + (a.blocks ? a.block_size : 0);
  auto it = shapes_.find(key);
  if (it == shapes_.end() && TuningEnabled()) {
    fg_pcg_shape sh{};
    sh.items = a.kp;
    sh.precision = a.precision;
    sh.block_size = a.blocks ? a.block_size : 0;
    // Candidates: 512-thread CTAs with the ring on / off (only 16-byte item vectors of
    // per-item operators can use it) x column cache off / on, and 1024-thread CTAs with the
    // ring (FP64 Jacobi, where the launch admits them).  Each runs kTuneIterations CG
    // iterations of this very system (tolerance 0: no item stops early); the real launch
    // follows and overwrites every vector the timing runs wrote.
    const int iv = a.precision == 0 ? (a.kp >= 2 ? 2 : 1) : (a.kp >= 4 ? 4 : (a.kp >= 2 ? 2 : 1));
    const bool ring_possible = (a.precision == 0 ? 8 : 4) * iv == 16 && a.value_item;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      cudaGetLastError();
      if (e0)
        cudaEventDestroy(e0);
      return cudaErrorUnknown;
    }
    // One untimed launch first (cold caches and clocks would favour whichever candidate
    // runs later), then kTuneRounds interleaved rounds; each candidate keeps its fastest.
    PcgArgs t = a;
    t.tolerance = 0.0;
    t.item_tolerance = nullptr;
    t.max_iterations = kTuneIterations;
    t.trace = nullptr;
    t.block_request = 2;
    if (LaunchPcg(t, nullptr, nullptr, stream) != cudaSuccess)
      cudaGetLastError();
    else
      timing_.kernel_launches += 1;
    for (int round = 0; round < kTuneRounds; ++round)
      for (int c = 0; c < 5; ++c) {
        const int ring = c % 2 == 0 ? 1 : 2, cache = c == 2 || c == 3 ? 1 : 2;
        if (ring == 1 && !ring_possible)
          continue;
        t.ring_request = ring;
        t.col_cache_request = cache;
        t.block_request = c == 4 ? 1 : 2;
        float ms = 0.0f;
        int threads = 0;
        if (cudaEventRecord(e0, stream) != cudaSuccess || LaunchPcg(t, nullptr, &threads, stream) != cudaSuccess ||
            cudaEventRecord(e1, stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
          cudaGetLastError();
          continue;
        }
        timing_.kernel_launches += 1;
        if (c == 4 && threads != 1024)
          continue; // the launch fell back to 512 threads: not a candidate of its own
        const double us = 1e3 * ms / kTuneIterations;
        if (sh.us_per_iteration[c] == 0.0) {
          ++sh.candidates;
          sh.us_per_iteration[c] = us;
        } else if (us < sh.us_per_iteration[c]) {
          sh.us_per_iteration[c] = us;
        }
      }
    double best = 0.0;
    for (int c = 0; c < 5; ++c)
      if (sh.us_per_iteration[c] > 0.0 && (best == 0.0 || sh.us_per_iteration[c] < best)) {
        best = sh.us_per_iteration[c];
        sh.value_ring = c % 2 == 0 ? 1 : 0;
        sh.column_cache = c == 2 || c == 3 ? 1 : 0;
        sh.threads_per_block = c == 4 ? 1024 : 512;
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (sh.candidates > 0)
      it = shapes_.emplace(key, sh).first;
  }
  if (it != shapes_.end()) {
    a.ring_request = it->second.value_ring ? 1 : 2;
    a.col_cache_request = it->second.column_cache ? 1 : 2;
    a.block_request = it->second.threads_per_block == 1024 ? 1 : 2;
  }
  return LaunchPcg(a, grid, block, stream);
}

Status Plan::BuildBlocks(int kp, int items, bool per_item, bool single, cudaStream_t stream)
{
  const int bs = block_size();
  if (!bs)
    return Status::kOk;
  if (LaunchBlockInverse(dev_, kp, items, bs, values_.get(), per_item ? 1 : 0, diag_.get(),
                         per_item ? 1 : 0, single ? nullptr : blocks64_.get(),
                         single ? blocks32_.get() : nullptr, block_fallbacks_.get(),
                         stream) != cudaSuccess) {
    cudaGetLastError();
    return Status::kInternalError;
  }
  timing_.kernel_launches += 1;
  timing_.block_inverses += static_cast<int64_t>(host_.n_pad / bs) * (per_item ? items : 1);
  return Status::kOk;
}

Status Plan::LinearSolve(int kp, int items, uint32_t mask, double tolerance, int max_iterations,
                         cudaStream_t stream, double *linfo, bool final_tolerance)
{
  // From the iterate: solve J delta = d, d = rhs - J x0 (x0 = the current state's free
  // values), to ||d - J delta|| <= tol ||rhs|| (per-item tolerance tol ||rhs|| / ||d||),
  // then x = x0 + delta -- the reference's acceptance rule, a different starting point.
  // With final_tolerance (the exact inner tolerance in the relaxed Newton regime) tol is
  // kIterateFinalTightening times the reference's: a solve started at the iterate leaves
  // its remaining error in the smooth, slowly converging modes that the flux linkage
  // integrates, so at the same residual its flux differs from a zero-start solve's by
  // up to 3e-8 (measured on the rotor-stator sector); near convergence the defect is a
  // small fraction of ||rhs||, and the tighter target costs few extra iterations.
  const double *b = rhs_.get();
  const double *item_tol = nullptr;
  uint32_t solve = mask;
  double done[3 * kMaxItems];
  if (from_iterate_) {
    double *h = small_.get();
    if (LaunchStateToFree(dev_, kp, state_.get(), x0_.get(), stream) != cudaSuccess ||
        LaunchEquationResidual(dev_, kp, values_.get(), rhs_.get(), x0_.get(), d_.get(),
                               norm_partials_.get(), norms_.get(), stream) != cudaSuccess ||
        cudaMemcpyAsync(h, norms_.get(), sizeof(double) * 2 * kp, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return Status::kInternalError;
    timing_.kernel_launches += 3;
    std::vector<double> tol_i(kp, tolerance);
    for (int i = 0; i < items; ++i) {
      if (!((mask >> i) & 1u))
        continue;
      const double dn = std::sqrt(h[i]), bn = std::sqrt(h[kp + i]);
      const double target =
          final_tolerance ? std::max(kIterateFinalTightening * tolerance, std::min(tolerance, kIterateFinalFloor))
                          : tolerance;
      if (std::isfinite(dn) && std::isfinite(bn) && dn <= target * bn) {
        solve &= ~(1u << i); // the iterate already meets the linear tolerance
        done[3 * i] = ToInt(Status::kOk);
        done[3 * i + 1] = 0;
        done[3 * i + 2] = dn;
      } else if (std::isfinite(dn) && std::isfinite(bn) && dn > 0.0) {
        tol_i[i] = target * bn / dn;
      }
    }
    Status s = item_tol_.upload(tol_i.data(), kp, stream);
    if (s != Status::kOk)
      return s;
    b = d_.get();
    item_tol = item_tol_.get();
  }
  if (solve) {
    if (options_.precision == FG_PRECISION_MIXED) {
      Status s = MixedSolve(kp, items, solve, tolerance, max_iterations, stream, linfo, b, item_tol);
      if (s != Status::kOk)
        return s;
    } else {
      Status s = BuildBlocks(kp, items, true, false, stream);
      if (s == Status::kOk)
        s = RunPcg(kp, items, solve, tolerance, max_iterations, kp, 1, kp, 1, 1, stream,
                   block_size() ? blocks64_.get() : nullptr, b, item_tol);
      if (s != Status::kOk)
        return s;
      int32_t err = 0;
      if (cudaMemcpyAsync(linfo, pcg_info_.get(), sizeof(double) * 3 * kp, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
          cudaMemcpyAsync(&err, error_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
          cudaStreamSynchronize(stream) != cudaSuccess)
        return Status::kInternalError;
      if (err)
        return Status::kInternalError;
    }
  }
  if (from_iterate_) {
    if (LaunchAddCorrection(dev_, kp, solve, x0_.get(), x_.get(), x_.get(), stream) != cudaSuccess)
      return Status::kInternalError;
    timing_.kernel_launches += 1;
    for (int i = 0; i < items; ++i)
      if (((mask >> i) & 1u) && !((solve >> i) & 1u))
        std::copy(done + 3 * i, done + 3 * i + 3, linfo + 3 * i);
  }
  return Status::kOk;
}

// FP32 PCG inside FP64 defect correction, as one launch with reliable updates: SpMV,
// preconditioner and vectors in FP32 (dot products and scalars in FP64); the solution
// accumulates in FP64 and the residual is replaced by the FP64 true residual
// b - K x (FP64 operator) each time the recursive residual has fallen tenfold, keeping the
// search direction, so the Krylov space is not rebuilt as it is by restarted refinement.
// Acceptance is the reference's rule on the FP64 true residual.  Items the FP32 solve
// cannot finish (breakdown, non-finite, iteration budget) are solved again by the FP64
// PCG from x = 0.
Status Plan::MixedSolve(int kp, int items, uint32_t mask, double tolerance, int max_iterations,
                        cudaStream_t st, double *linfo, const double *b, const double *item_tol)
{
  constexpr double kReliableDelta = 0.1;
  if (LaunchToSingle(dev_, kp, mask, values_.get(), diag_.get(), v32_.get(), d32_.get(), i32_.get(),
                     st) != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 1;
  Status s = BuildBlocks(kp, items, true, true, st);
  if (s != Status::kOk)
    return s;
  PcgArgs a{};
  a.precision = 1;
  a.n = host_.n;
  a.n_pad = host_.n_pad;
  a.slices = host_.slices;
  a.kp = kp;
  a.items = items;
  a.slice_off = slice_off_.get();
  a.host_slice_off = host_.slice_off.data();
  a.row_len = row_len_.get();
  a.sell_col = sell_col_.get();
  a.values = v32_.get();
  a.value_stride = kp;
  a.value_item = 1;
  a.diag = d32_.get();
  a.invd = i32_.get();
  a.diag_stride = kp;
  a.diag_item = 1;
  a.use_inverse = 1;
  if (block_size()) {
    a.blocks = blocks32_.get();
    a.block_size = block_size();
    a.block_stride = kp;
    a.block_item = 1;
  }
  a.b = nullptr;
  a.x = x32_.get();
  a.r = r32_.get();
  a.z = z32_.get();
  a.p0 = p032_.get();
  a.p1 = p132_.get();
  a.q = q32_.get();
  a.reliable = 1;
  a.reliable_delta = kReliableDelta;
  a.values64 = values_.get();
  a.b64 = b;
  a.x64 = x_.get();
  a.partials = pcg_partials_.get();
  a.barrier = barrier_.get();
  a.error = error_.get();
  a.info = pcg_info_.get();
  a.tolerance = tolerance;
  a.item_tolerance = item_tol;
  a.max_iterations = max_iterations;
  a.active_mask = mask;
  a.timeout_ns = PcgWaitLimitNs();
  a.trace = trace_enabled_ ? trace_.get() : nullptr;
  int grid = 0, block = 0;
  if (LaunchShaped(a, &grid, &block, st) != cudaSuccess) {
    cudaGetLastError();
    return Status::kInternalError;
  }
  timing_.pcg_grid = grid;
  timing_.pcg_block = block;
  timing_.pcg_launches += 1;
  timing_.kernel_launches += 1;
  int32_t err = 0;
  if (cudaMemcpyAsync(linfo, pcg_info_.get(), sizeof(double) * 3 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(&err, error_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return Status::kInternalError;
  if (err)
    return Status::kInternalError;
  uint32_t fallback = 0;
  for (int i = 0; i < items; ++i) {
    if (!((mask >> i) & 1u))
      continue;
    const int status = static_cast<int>(linfo[3 * i]);
    if (status == ToInt(Status::kInvalidArgument))
      continue;
    if (status != ToInt(Status::kOk))
      fallback |= 1u << i;
  }
  if (fallback) {
    double first[3 * kMaxItems];
    std::copy(linfo, linfo + 3 * kp, first);
    if ((s = BuildBlocks(kp, items, true, false, st)) != Status::kOk ||
        (s = RunPcg(kp, items, fallback, tolerance, max_iterations, kp, 1, kp, 1, 1, st,
                    block_size() ? blocks64_.get() : nullptr, b, item_tol)) != Status::kOk)
      return s;
    if (cudaMemcpyAsync(linfo, pcg_info_.get(), sizeof(double) * 3 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&err, error_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return Status::kInternalError;
    if (err)
      return Status::kInternalError;
    for (int i = 0; i < items; ++i) {
      if ((fallback >> i) & 1u)
        linfo[3 * i + 1] += first[3 * i + 1];
      else
        std::copy(first + 3 * i, first + 3 * i + 3, linfo + 3 * i);
    }
    timing_.mixed_fallbacks += __builtin_popcount(fallback);
  }
  return Status::kOk;
}

Status Plan::SolveDevice(const SolveRequest &req)
{
  timing_ = fg_timing{};
  if (host_only_)
    return Status::kGpuUnavailable;
  if (req.items <= 0 || (!req.currents && host_.C > 0) || !req.info)
    return Status::kInvalidArgument;
  if (trace_enabled_ &&
      cudaMemsetAsync(trace_.get(), 0, sizeof(unsigned long long) * kPcgTraceSlots, req.stream) != cudaSuccess)
    return Status::kInternalError;
  if (block_fallbacks_.get() &&
      cudaMemsetAsync(block_fallbacks_.get(), 0, sizeof(int32_t), req.stream) != cudaSuccess)
    return Status::kInternalError;
  if (ChunksTogether(req)) {
    // Waves of at most kMaxLanes chunks (fewer when device memory is short, or when their
    // vectors would not fit L2 together), balanced; a wave of one is a chunk on its own.
    const int total = (req.items + chunk_cap_ - 1) / chunk_cap_;
    Status s = EnsureWorkspace(kMaxItems);
    if (s != Status::kOk)
      return s;
    size_t free_bytes = 0, total_bytes = 0;
    int cap = kMaxLanes;
    if (cudaMemGetInfo(&free_bytes, &total_bytes) == cudaSuccess) {
      const size_t lane = std::max<size_t>(DeviceBytes(), 1);
      const size_t fit = static_cast<size_t>(lanes_.size()) + 1 + free_bytes / 2 / lane;
      cap = static_cast<int>(std::max<size_t>(1, std::min<size_t>(kMaxLanes, fit)));
    } else {
      cudaGetLastError();
    }
    // Chunks advance together only while their vectors fit half of L2 together: beyond
    // that every CG iteration streams them from HBM, and a chunk alone (whose vectors stay
    // in L2 while the operator values stream past) is faster.  Measured on the 40k-node
    // rotor-stator sector (62 MB of vectors per chunk): 32 chunks together ran at 0.44x the
    // chunk-after-chunk rate.
    int device = 0, l2 = 0;
    if (ChunksTogetherMode() == 1 && cudaGetDevice(&device) == cudaSuccess &&
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device) == cudaSuccess && l2 > 0) {
      const size_t fit = static_cast<size_t>(l2) / 2 / std::max<size_t>(ChunkVectorBytes(host_.n_pad), 1);
      cap = std::min(cap, static_cast<int>(std::max<size_t>(1, fit)));
    }
    const int waves = (total + cap - 1) / cap;
    const int per_wave = (total + waves - 1) / waves;
    for (int c0 = 0; c0 < total; c0 += per_wave) {
      const int n = std::min(per_wave, total - c0);
      const int first = c0 * chunk_cap_;
      s = n > 1 ? SolveChunksTogether(req, first, n) : SolveChunk(req, first, std::min(chunk_cap_, req.items - first));
      if (s != Status::kOk)
        return s;
    }
  } else {
    for (int first = 0; first < req.items; first += chunk_cap_) {
      const Status s = SolveChunk(req, first, std::min(chunk_cap_, req.items - first));
      if (s != Status::kOk)
        return s;
    }
  }
  if (block_size()) {
    int32_t fallbacks = 0;
    if (cudaMemcpyAsync(&fallbacks, block_fallbacks_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost,
                        req.stream) != cudaSuccess ||
        cudaStreamSynchronize(req.stream) != cudaSuccess)
      return Status::kInternalError;
    timing_.block_fallbacks = fallbacks;
  }
  if (trace_enabled_) {
    unsigned long long t[kPcgTraceSlots];
    if (cudaMemcpy(t, trace_.get(), sizeof(t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return Status::kInternalError;
    for (int s = 0; s < 9; ++s)
      timing_.pcg_phase_ms[s] = static_cast<double>(t[s]) * 1e-6;
    timing_.pcg_phase_ms[9] = static_cast<double>(t[9]);
  }
  return Status::kOk;
}

bool Plan::ChunksTogether(const SolveRequest &req) const
{
  return ChunksTogetherMode() != 0 && req.items > chunk_cap_ && chunk_cap_ == kMaxItems &&
         options_.precision == FG_PRECISION_FP64 && block_size() == 0 && !from_iterate_ && !one_reduction_ &&
         !req.guard_warm &&
         !trace_enabled_ && MultiPcgMaxGrid(kMaxItems) > 0;
}

Status Plan::EnsureLanes(int lanes)
{
  while (static_cast<int>(lanes_.size()) + 1 < lanes) {
    // A lane: this plan's host model and plan, its own device constants and workspace.
    auto lane = std::make_unique<Plan>();
    lane->model_ = model_;
    lane->host_ = host_;
    lane->options_ = options_;
    lane->options_.flags |= FG_PLAN_HOST_ONLY;
    lane->chunk_cap_ = chunk_cap_;
    lane->from_iterate_ = from_iterate_;
    lane->host_only_ = true;
    Status s = lane->AttachDevice();
    if (s != Status::kOk)
      return s;
    lanes_.push_back(std::move(lane));
  }
  if (!lane_solver_ || lane_solver_lanes_ != lanes) {
    std::vector<Plan *> plans{this};
    for (int i = 0; i + 1 < lanes; ++i)
      plans.push_back(lanes_[i].get());
    auto solver = std::make_unique<MultiSolver>();
    const Status s = solver->Create(plans, kMaxItems);
    if (s != Status::kOk)
      return s;
    lane_solver_ = std::move(solver);
    lane_solver_lanes_ = lanes;
  }
  return Status::kOk;
}

Status Plan::SolveChunksTogether(const SolveRequest &req, int first, int chunks)
{
  std::vector<int> firsts, counts;
  for (int c = 0; c < chunks; ++c) {
    const int f = first + c * chunk_cap_;
    firsts.push_back(f);
    counts.push_back(std::min(chunk_cap_, req.items - f));
  }
  Status s = EnsureLanes(chunks);
  if (s != Status::kOk)
    return s;
  const fg_timing before = timing_;
  s = lane_solver_->SolveChunks(req, firsts, counts);
  // Every lane's own counters (this plan's included) were reset by the lock-step solve.
  fg_timing lanes_sum{};
  for (int i = 0; i < chunks; ++i) {
    const fg_timing &t = i == 0 ? timing_ : lanes_[i - 1]->timing_;
    lanes_sum.pcg_iterations += t.pcg_iterations;
    lanes_sum.kernel_launches += t.kernel_launches;
  }
  const fg_multi_timing &mt = lane_solver_->timing();
  timing_ = before;
  timing_.pcg_iterations += lanes_sum.pcg_iterations;
  timing_.kernel_launches += lanes_sum.kernel_launches + mt.pcg_launches;
  timing_.pcg_launches += mt.pcg_launches;
  timing_.newton_iterations += mt.newton_steps;
  return s;
}

Status Plan::SolveChunk(const SolveRequest &req, int first, int k)
{
  Chunk c;
  Status s = ChunkBegin(req, first, k, &c);
  if (s != Status::kOk || !c.valid)
    return s;
  while (c.iteration < req.options.max_newton_iterations && c.active) {
    if ((s = ChunkAssemble(&c)) != Status::kOk || (s = ChunkLinear(&c)) != Status::kOk ||
        (s = ChunkNorms(&c, false)) != Status::kOk)
      return s;
    if (cudaStreamSynchronize(req.stream) != cudaSuccess)
      return Status::kInternalError;
    if ((s = ChunkDecide(&c)) != Status::kOk || (s = ChunkUpdate(&c)) != Status::kOk)
      return s;
  }
  if ((s = ChunkRecover(&c)) != Status::kOk)
    return s;
  return ChunkFinish(&c);
}

Status Plan::ChunkBegin(const SolveRequest &req, int first, int k, Chunk *c, int min_kp)
{
  const fg_solve_options &o = req.options;
  const int N = host_.N, C = host_.C;
  cudaStream_t st = req.stream;
  c->req = &req;
  c->first = first;
  c->k = k;
  c->valid = false;
  for (int i = 0; i < k; ++i) {
    fg_item_info &inf = req.info[first + i];
    inf = fg_item_info{};
    inf.status = ToInt(Status::kInvalidArgument);
    inf.residual_l2 = std::numeric_limits<double>::infinity();
    inf.last_linear_tolerance = std::numeric_limits<double>::quiet_NaN();
    inf.verified_equation_residual_relative = std::numeric_limits<double>::infinity();
  }
  if (!(o.relative_tolerance > 0.0) || !std::isfinite(o.relative_tolerance) ||
      o.max_newton_iterations < 0 || o.max_linear_iterations < 0)
    return Status::kOk; // per-item INVALID_ARGUMENT, as SolveBatch returns
  const int kp = std::max(PadItems(k), PadItems(min_kp));
  c->kp = kp;
  Status s = EnsureWorkspace(kp);
  if (s != Status::kOk)
    return s;
  c->currents = req.currents + static_cast<size_t>(first) * C;
  c->hc = req.hc_scale ? req.hc_scale + first : nullptr;
  const double *warm = req.warm ? req.warm + static_cast<size_t>(first) * N : nullptr;

  // Non-finite currents make an item invalid before any work (nonlinear_solver.cu:198-206).
  uint32_t active = 0;
  {
    std::vector<double> cur(static_cast<size_t>(k) * C);
    if (C > 0 && cudaMemcpyAsync(cur.data(), c->currents, cur.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return Status::kInternalError;
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return Status::kInternalError;
    for (int i = 0; i < k; ++i) {
      bool finite = true;
      for (int j = 0; j < C; ++j)
        finite = finite && std::isfinite(cur[static_cast<size_t>(i) * C + j]);
      if (finite)
        active |= 1u << i;
    }
  }
  c->adaptive = o.adaptive_linear_tolerance != 0 && host_.has_nonlinear;
  uint32_t warm_mask = warm ? active : 0u;
  if (warm && req.guard_warm && active) {
    // Equation residual ||K(A) A - b|| at the zero start and at the warm start; an item
    // keeps its warm start only if the residual there is smaller.
    double res[2][kMaxItems];
    for (int pass = 0; pass < 2; ++pass) {
      if (LaunchInitState(dev_, kp, warm, k, pass ? active : 0u, state_.get(), st) != cudaSuccess ||
          cudaMemsetAsync(invalid_.get(), 0, sizeof(int32_t) * kp, st) != cudaSuccess ||
          LaunchElementKernel(dev_, kp, state_.get(), active, active, ev_.get(), er_.get(),
                              invalid_.get(), st) != cudaSuccess ||
          LaunchGatherValues(dev_, kp, ev_.get(), active, values_.get(), diag_.get(), invd_.get(),
                             invalid_.get(), st) != cudaSuccess ||
          LaunchGatherRhs(dev_, kp, er_.get(), c->currents, c->hc, active, rhs_.get(), st) != cudaSuccess ||
          LaunchStateToFree(dev_, kp, state_.get(), x0_.get(), st) != cudaSuccess ||
          LaunchEquationResidual(dev_, kp, values_.get(), rhs_.get(), x0_.get(), nullptr,
                                 norm_partials_.get(), norms_.get(), st) != cudaSuccess ||
          cudaMemcpyAsync(small_.get(), norms_.get(), sizeof(double) * 2 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        return Status::kInternalError;
      timing_.kernel_launches += 8;
      for (int i = 0; i < k; ++i)
        res[pass][i] = std::sqrt(small_.get()[i]);
    }
    for (int i = 0; i < k; ++i)
      if (((active >> i) & 1u) && !(res[1][i] < res[0][i]))
        warm_mask &= ~(1u << i);
  }
  for (int i = 0; i < k; ++i)
    if (warm)
      req.info[first + i].warm_start = ((warm_mask >> i) & 1u) ? 1 : 2;
  if (LaunchInitState(dev_, kp, warm, k, warm_mask, state_.get(), st) != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 1;
  c->active = active;
  c->warm_mask = warm_mask;
  c->relax.assign(k, 1.0);
  c->prev.assign(k, std::numeric_limits<double>::infinity());
  c->iteration = 0;
  c->valid = true;
  return Status::kOk;
}

// The inner tolerance of this Newton step: the tightest of the active items'
// (BatchNewtonLinearTolerance, nonlinear_model.cpp:176-184).
void Plan::ChunkTolerance(Chunk *c)
{
  const fg_solve_options &o = c->req->options;
  c->tol = std::numeric_limits<double>::infinity();
  for (int i = 0; i < c->k; ++i)
    if ((c->active >> i) & 1u)
      c->tol = std::min(c->tol, NewtonLinearTolerance(o, c->adaptive, c->prev[i]));
}

// Enqueues the Newton system of the active items at the current state.
Status Plan::ChunkAssemble(Chunk *c)
{
  cudaStream_t st = c->req->stream;
  const int kp = c->kp;
  ChunkTolerance(c);
  // Iteration 0 of a cold start uses the cold secant; a warm start is Newton from the
  // first iteration (nonlinear_solver.cu:698).
  const uint32_t newton_mask = c->iteration > 0 ? c->active : (c->active & c->warm_mask);
  if (c->timed)
    cudaEventRecord(ev_start_, st);
  if (cudaMemsetAsync(invalid_.get(), 0, sizeof(int32_t) * kp, st) != cudaSuccess ||
      LaunchElementKernel(dev_, kp, state_.get(), newton_mask, c->active, ev_.get(), er_.get(),
                          invalid_.get(), st) != cudaSuccess ||
      LaunchGatherValues(dev_, kp, ev_.get(), c->active, values_.get(), diag_.get(), invd_.get(),
                         invalid_.get(), st) != cudaSuccess ||
      LaunchGatherRhs(dev_, kp, er_.get(), c->currents, c->hc, c->active, rhs_.get(), st) != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 3;
  if (c->timed)
    cudaEventRecord(ev_mid_, st);
  return Status::kOk;
}

bool Plan::ChunkPcgArgs(const Chunk &c, unsigned *barrier, int32_t *error, PcgArgs *out)
{
  if (options_.precision != FG_PRECISION_FP64 || block_size() != 0 || from_iterate_ || one_reduction_)
    return false;
  PcgArgs a{};
  a.n = host_.n;
  a.n_pad = host_.n_pad;
  a.slices = host_.slices;
  a.kp = c.kp;
  a.items = c.k;
  a.slice_off = slice_off_.get();
  a.row_len = row_len_.get();
  a.sell_col = sell_col_.get();
  a.values = values_.get();
  a.value_stride = c.kp;
  a.value_item = 1;
  a.diag = diag_.get();
  a.invd = invd_.get();
  a.diag_stride = c.kp;
  a.diag_item = 1;
  a.use_inverse = 1;
  a.b = rhs_.get();
  a.x = x_.get();
  a.r = r_.get();
  a.z = z_.get();
  a.p0 = p0_.get();
  a.p1 = p1_.get();
  a.q = q_.get();
  a.partials = pcg_partials_.get();
  a.barrier = barrier;
  a.error = error;
  a.info = pcg_info_.get();
  a.tolerance = c.tol;
  a.max_iterations = c.req->options.max_linear_iterations;
  a.active_mask = c.active;
  a.timeout_ns = PcgWaitLimitNs();
  *out = a;
  return true;
}

Status Plan::ChunkLinear(Chunk *c)
{
  // The tighter iterate-start target applies where the answer can be returned (the exact
  // inner tolerance) after the reference's first five undamped steps: a Newton that runs
  // into the relaxed regime (saturated iron) carries the candidate's smooth-mode solve error
  // into its answer; workloads converging within five steps meet the flux bound without it.
  const bool tighten = c->tol <= c->req->options.linear_relative_tolerance && c->iteration > 5;
  Status s = LinearSolve(c->kp, c->k, c->active, c->tol, c->req->options.max_linear_iterations,
                         c->req->stream, c->linfo, tighten);
  if (s == Status::kOk && c->timed)
    cudaEventRecord(ev_pcg_, c->req->stream);
  return s;
}

// Step norms and the small summary back to the host (asynchronously, into small_):
// PCG info [3kp] (copied from the device when linfo_on_device), norms [2kp], assembly
// flags, the PCG error flag.
Status Plan::ChunkNorms(Chunk *c, bool linfo_on_device)
{
  cudaStream_t st = c->req->stream;
  const int kp = c->kp;
  double *h = small_.get();
  if (LaunchNewtonNorms(dev_, kp, x_.get(), state_.get(), norm_partials_.get(), norms_.get(), st) !=
      cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 2;
  if (linfo_on_device) {
    if (cudaMemcpyAsync(h, pcg_info_.get(), sizeof(double) * 3 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return Status::kInternalError;
  } else {
    std::memcpy(h, c->linfo, sizeof(double) * 3 * kp);
  }
  if (cudaMemcpyAsync(h + 3 * kp, norms_.get(), sizeof(double) * 2 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(reinterpret_cast<int32_t *>(h + 5 * kp), invalid_.get(), sizeof(int32_t) * kp,
                      cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(reinterpret_cast<int32_t *>(h + 6 * kp), error_.get(), sizeof(int32_t),
                      cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return Status::kInternalError;
  return Status::kOk;
}

// Host Newton policy after the summary has arrived: statuses, relaxation, the step gate.
Status Plan::ChunkDecide(Chunk *c)
{
  const fg_solve_options &o = c->req->options;
  const int kp = c->kp, k = c->k;
  const double *h = small_.get();
  if (c->timed) {
    timing_.assembly_ms += Elapsed(ev_start_, ev_mid_);
    timing_.pcg_ms += Elapsed(ev_mid_, ev_pcg_);
  }
  timing_.newton_iterations += 1;
  const double *pinfo = h, *norms = h + 3 * kp;
  const int32_t *invalid = reinterpret_cast<const int32_t *>(h + 5 * kp);
  const int32_t pcg_error = *reinterpret_cast<const int32_t *>(h + 6 * kp);
  if (pcg_error != 0)
    return Status::kInternalError;
  int max_its = 0;
  c->rel = ItemScalars{};
  c->update = 0;
  const uint32_t was_active = c->active;
  for (int i = 0; i < k; ++i) {
    if (!((was_active >> i) & 1u))
      continue;
    fg_item_info &inf = c->req->info[c->first + i];
    if (invalid[i]) {
      inf.status = ToInt(Status::kAssemblyFailed);
      c->active &= ~(1u << i);
      continue;
    }
    const int pstatus = static_cast<int>(pinfo[3 * i]);
    const int pits = static_cast<int>(pinfo[3 * i + 1]);
    max_its = std::max(max_its, pits);
    inf.linear_iterations += pits;
    inf.last_linear_tolerance = c->tol;
    if (pstatus != 0) {
      inf.status = pstatus;
      inf.iterations = pits;
      inf.residual_l2 = pinfo[3 * i + 2];
      c->active &= ~(1u << i);
      continue;
    }
    const double dd = norms[i], cc = norms[kp + i];
    const double residual = std::sqrt(dd) / std::max(std::sqrt(cc), std::numeric_limits<double>::min());
    inf.iterations = c->iteration + 1;
    inf.residual_l2 = residual;
    if (!std::isfinite(residual)) {
      inf.status = ToInt(Status::kNumericalNonfinite);
      c->active &= ~(1u << i);
      continue;
    }
    if (c->iteration > 5) {
      if (residual > c->prev[i] && c->relax[i] > 0.125)
        c->relax[i] *= 0.5;
      else
        c->relax[i] += 0.1 * (1.0 - c->relax[i]);
    }
    c->rel.v[i] = c->relax[i];
    c->update |= 1u << i;
    if (c->iteration > 0 && residual < 100.0 * o.relative_tolerance && c->tol <= o.linear_relative_tolerance) {
      inf.status = ToInt(Status::kOk);
      c->active &= ~(1u << i);
    } else {
      c->prev[i] = residual;
    }
  }
  timing_.pcg_iterations += max_its;
  return Status::kOk;
}

Status Plan::ChunkUpdate(Chunk *c)
{
  cudaStream_t st = c->req->stream;
  if (c->update && LaunchNewtonUpdate(dev_, c->kp, x_.get(), state_.get(), c->rel, c->update, st) != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += c->update ? 1 : 0;
  ++c->iteration;
  return Status::kOk;
}

// Equation residual ||J x0 - rhs|| and ||rhs|| of the items in mask at the current state
// (the system must have been assembled there); res[i] receives the first, for all kp.
Status Plan::EquationNorms(int kp, cudaStream_t st, double *res)
{
  if (LaunchStateToFree(dev_, kp, state_.get(), x0_.get(), st) != cudaSuccess ||
      LaunchEquationResidual(dev_, kp, values_.get(), rhs_.get(), x0_.get(), nullptr, norm_partials_.get(),
                             norms_.get(), st) != cudaSuccess ||
      cudaMemcpyAsync(small_.get() + 8 * kp, norms_.get(), sizeof(double) * 2 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(reinterpret_cast<int32_t *>(small_.get() + 7 * kp), invalid_.get(), sizeof(int32_t) * kp,
                      cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 3;
  for (int i = 0; i < kp; ++i)
    res[i] = std::sqrt(small_.get()[8 * kp + i]);
  return Status::kOk;
}

// SolveSafeguarded (gpu_solver/src/solvers/nonlinear_solver.cu:534-659) for the items the
// Newton loop exhausted, when the options ask for recovery (:515-530): from the zero start,
// undamped Newton directions at the fixed linear tolerance, each accepted through Armijo
// backtracking (at most 20 halvings, sufficient decrease 1e-4) on the equation residual
// ||K(A) A - b||; done when the step is below 100 x relative_tolerance and the residual
// has fallen by relative_tolerance.  The zero start already holds the expanded fixed
// values, so the reference's root expansion before the first direction changes nothing.
Status Plan::ChunkRecover(Chunk *c)
{
  const fg_solve_options &o = c->req->options;
  const uint32_t rec = c->active;
  if (!o.recover_nonconvergence || o.max_newton_iterations <= 0 || !rec)
    return Status::kOk;
  cudaStream_t st = c->req->stream;
  const int kp = c->kp, k = c->k;
  const double rel = o.relative_tolerance;
  std::vector<int32_t> orig_its(k), orig_lin(k);
  for (int i = 0; i < k; ++i) {
    fg_item_info &inf = c->req->info[c->first + i];
    orig_its[i] = inf.iterations;
    orig_lin[i] = inf.linear_iterations;
    if ((rec >> i) & 1u) {
      inf.status = ToInt(Status::kNonlinearSolveNotConverged);
      inf.iterations = 0;
      inf.linear_iterations = 0;
      inf.residual_l2 = std::numeric_limits<double>::infinity();
    }
  }
  c->active &= ~rec;
  auto assemble = [&](uint32_t mask) {
    return cudaMemsetAsync(invalid_.get(), 0, sizeof(int32_t) * kp, st) == cudaSuccess &&
           LaunchElementKernel(dev_, kp, state_.get(), mask, mask, ev_.get(), er_.get(), invalid_.get(), st) ==
               cudaSuccess &&
           LaunchGatherValues(dev_, kp, ev_.get(), mask, values_.get(), diag_.get(), invd_.get(), invalid_.get(),
                              st) == cudaSuccess &&
           LaunchGatherRhs(dev_, kp, er_.get(), c->currents, c->hc, mask, rhs_.get(), st) == cudaSuccess;
  };
  const int32_t *invalid = reinterpret_cast<const int32_t *>(small_.get() + 7 * kp);
  std::vector<double> norm(kp, 0.0), scale(kp, 1.0), res(kp, 0.0);
  if (LaunchResetState(dev_, kp, rec, state_.get(), st) != cudaSuccess || !assemble(rec))
    return Status::kInternalError;
  timing_.kernel_launches += 4;
  Status s = EquationNorms(kp, st, res.data());
  if (s != Status::kOk)
    return s;
  uint32_t run = rec;
  for (int i = 0; i < k; ++i)
    if ((rec >> i) & 1u) {
      if (invalid[i]) {
        c->req->info[c->first + i].status = ToInt(Status::kAssemblyFailed);
        run &= ~(1u << i);
      }
      norm[i] = res[i];
      scale[i] = std::max(norm[i], std::numeric_limits<double>::min());
    }
  for (int iteration = 0; iteration < o.max_newton_iterations && run; ++iteration) {
    for (int i = 0; i < k; ++i)
      if (((run >> i) & 1u) && !std::isfinite(norm[i])) {
        c->req->info[c->first + i].status = ToInt(Status::kNumericalNonfinite);
        run &= ~(1u << i);
      }
    if (!run)
      break;
    double linfo[3 * kMaxItems];
    if ((s = LinearSolve(kp, k, run, o.linear_relative_tolerance, o.max_linear_iterations, st, linfo)) != Status::kOk)
      return s;
    double *h = small_.get();
    if (LaunchNewtonNorms(dev_, kp, x_.get(), state_.get(), norm_partials_.get(), norms_.get(), st) != cudaSuccess ||
        cudaMemcpyAsync(h, norms_.get(), sizeof(double) * 2 * kp, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return Status::kInternalError;
    timing_.kernel_launches += 2;
    timing_.newton_iterations += 1;
    uint32_t trying = 0;
    for (int i = 0; i < k; ++i) {
      if (!((run >> i) & 1u))
        continue;
      fg_item_info &inf = c->req->info[c->first + i];
      inf.linear_iterations += static_cast<int32_t>(linfo[3 * i + 1]);
      inf.last_linear_tolerance = o.linear_relative_tolerance;
      if (static_cast<int>(linfo[3 * i]) != 0) {
        inf.status = static_cast<int>(linfo[3 * i]);
        inf.iterations = static_cast<int32_t>(linfo[3 * i + 1]);
        inf.residual_l2 = linfo[3 * i + 2];
        continue;
      }
      const double step = std::sqrt(h[i]) / std::max(std::sqrt(h[kp + i]), std::numeric_limits<double>::min());
      inf.iterations = iteration + 1;
      inf.residual_l2 = step;
      if (!std::isfinite(step)) {
        inf.status = ToInt(Status::kNumericalNonfinite);
        continue;
      }
      if (step < 100.0 * rel && norm[i] / scale[i] <= rel) {
        inf.status = ToInt(Status::kOk);
        continue;
      }
      trying |= 1u << i;
    }
    run = trying;
    if (!trying)
      break;
    // Armijo backtracking from the saved state along the undamped direction.
    if (LaunchMaskedCopy(dev_, kp, trying, state_.get(), saved_.get(), st) != cudaSuccess)
      return Status::kInternalError;
    ItemScalars alpha{};
    for (int i = 0; i < k; ++i)
      alpha.v[i] = 1.0;
    uint32_t accepted = 0;
    for (int backtrack = 0; backtrack < 20 && trying; ++backtrack) {
      if (LaunchTrial(dev_, kp, x_.get(), saved_.get(), state_.get(), alpha, trying, st) != cudaSuccess ||
          !assemble(trying))
        return Status::kInternalError;
      timing_.kernel_launches += 4;
      if ((s = EquationNorms(kp, st, res.data())) != Status::kOk)
        return s;
      for (int i = 0; i < k; ++i) {
        if (!((trying >> i) & 1u))
          continue;
        if (invalid[i]) {
          c->req->info[c->first + i].status = ToInt(Status::kAssemblyFailed);
          trying &= ~(1u << i);
          run &= ~(1u << i);
          continue;
        }
        const double trial = res[i];
        if (std::isfinite(trial) &&
            (trial <= (1.0 - 1e-4 * alpha.v[i]) * norm[i] || trial / scale[i] <= rel)) {
          norm[i] = trial;
          accepted |= 1u << i;
          trying &= ~(1u << i);
        } else {
          alpha.v[i] *= 0.5;
        }
      }
    }
    // Not accepted after 20 halvings: back to the last accepted state; recovery stops.
    if (trying && LaunchMaskedCopy(dev_, kp, trying, saved_.get(), state_.get(), st) != cudaSuccess)
      return Status::kInternalError;
    run = accepted;
  }
  for (int i = 0; i < k; ++i)
    if ((rec >> i) & 1u) {
      fg_item_info &inf = c->req->info[c->first + i];
      inf.iterations += orig_its[i];
      inf.linear_iterations += orig_lin[i];
      inf.verified_equation_residual_relative = norm[i] / scale[i];
    }
  return cudaStreamSynchronize(st) == cudaSuccess ? Status::kOk : Status::kInternalError;
}

Status Plan::ChunkFinish(Chunk *c)
{
  const SolveRequest &req = *c->req;
  const int N = host_.N, E = host_.E, C = host_.C, k = c->k, first = c->first;
  cudaStream_t st = req.stream;
  for (int i = 0; i < k; ++i)
    if ((c->active >> i) & 1u)
      req.info[first + i].status = ToInt(Status::kNonlinearSolveNotConverged);
  if (c->timed)
    cudaEventRecord(ev_mid_, st);
  const cudaError_t fe = LaunchFinalize(
      dev_, c->kp, k, state_.get(), req.a_out ? req.a_out + static_cast<size_t>(first) * N : nullptr,
      req.b1_out ? req.b1_out + static_cast<size_t>(first) * E : nullptr,
      req.b2_out ? req.b2_out + static_cast<size_t>(first) * E : nullptr,
      req.flux_out ? req.flux_out + static_cast<size_t>(first) * C : nullptr, st);
  if (fe != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 3;
  if (c->timed) {
    cudaEventRecord(ev_pcg_, st);
    if (cudaStreamSynchronize(st) != cudaSuccess)
      return Status::kInternalError;
    timing_.finalize_ms += Elapsed(ev_mid_, ev_pcg_);
  }
  return Status::kOk;
}

Status Plan::SolveHost(int items, const double *currents, const double *hc_scale,
                       const double *warm, const fg_solve_options &options, double *a_out,
                       double *b1_out, double *b2_out, double *flux_out, fg_item_info *info,
                       const double *warm_device, bool guard_warm)
{
  if (host_only_)
    return Status::kGpuUnavailable;
  if (items <= 0 || (!currents && host_.C > 0) || !info)
    return Status::kInvalidArgument;
  const size_t N = host_.N, E = host_.E, C = host_.C, k = items;
  Status s = Status::kOk;
  if ((s = in_currents_.upload(currents, k * C)) != Status::kOk)
    return s;
  if (hc_scale && (s = in_hc_.upload(hc_scale, k)) != Status::kOk)
    return s;
  if (warm && (s = in_warm_.upload(warm, k * N)) != Status::kOk)
    return s;
  if ((a_out && (s = out_a_.ensure(k * N)) != Status::kOk) ||
      (b1_out && (s = out_b1_.ensure(k * E)) != Status::kOk) ||
      (b2_out && (s = out_b2_.ensure(k * E)) != Status::kOk) ||
      (flux_out && (s = out_flux_.ensure(k * C)) != Status::kOk))
    return s;
  SolveRequest req;
  req.items = items;
  req.currents = in_currents_.get();
  req.hc_scale = hc_scale ? in_hc_.get() : nullptr;
  req.warm = warm_device ? warm_device : (warm ? in_warm_.get() : nullptr);
  req.guard_warm = guard_warm;
  req.options = options;
  req.a_out = a_out ? out_a_.get() : nullptr;
  req.b1_out = b1_out ? out_b1_.get() : nullptr;
  req.b2_out = b2_out ? out_b2_.get() : nullptr;
  req.flux_out = flux_out ? out_flux_.get() : nullptr;
  req.info = info;
  req.stream = nullptr;
  s = SolveDevice(req);
  if (s != Status::kOk)
    return s;
  if ((a_out && cudaMemcpy(a_out, out_a_.get(), k * N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (b1_out && cudaMemcpy(b1_out, out_b1_.get(), k * E * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (b2_out && cudaMemcpy(b2_out, out_b2_.get(), k * E * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (flux_out && C > 0 && cudaMemcpy(flux_out, out_flux_.get(), k * C * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
    return Status::kInternalError;
  return Status::kOk;
}

Status Plan::Assemble(int items, const double *states, const double *currents,
                      const int32_t *use_newton, double *values, double *diagonal, double *rhs)
{
  if (host_only_)
    return Status::kGpuUnavailable;
  if (items <= 0 || items > kMaxItems || !states || (!currents && host_.C > 0) || !use_newton)
    return Status::kInvalidArgument;
  const int kp = PadItems(items);
  Status s = EnsureWorkspace(kp);
  if (s != Status::kOk)
    return s;
  const size_t N = host_.N, C = host_.C, n = host_.n, nnz = host_.nnz;
  if ((s = in_warm_.upload(states, items * N)) != Status::kOk ||
      (s = in_currents_.upload(currents, items * C)) != Status::kOk ||
      (s = staging_.ensure(nnz + 2 * n)) != Status::kOk)
    return s;
  uint32_t newton = 0, active = 0;
  for (int i = 0; i < items; ++i) {
    active |= 1u << i;
    if (use_newton[i])
      newton |= 1u << i;
  }
  if (LaunchInterleave(kp, items, static_cast<int>(N), static_cast<int>(N), in_warm_.get(), state_.get(), nullptr) != cudaSuccess ||
      cudaMemset(invalid_.get(), 0, sizeof(int32_t) * kp) != cudaSuccess ||
      LaunchElementKernel(dev_, kp, state_.get(), newton, active, ev_.get(), er_.get(), invalid_.get(), nullptr) != cudaSuccess ||
      LaunchGatherValues(dev_, kp, ev_.get(), active, values_.get(), diag_.get(), invd_.get(), invalid_.get(), nullptr) != cudaSuccess ||
      LaunchGatherRhs(dev_, kp, er_.get(), in_currents_.get(), nullptr, active, rhs_.get(), nullptr) != cudaSuccess)
    return Status::kInternalError;
  std::vector<int32_t> invalid(kp);
  for (int i = 0; i < items; ++i) {
    double *sv = staging_.get(), *sd = sv + nnz, *sr = sd + n;
    if (LaunchExtractCsr(dev_, kp, i, values_.get(), diag_.get(), rhs_.get(), sv, sd, sr, nullptr) != cudaSuccess)
      return Status::kInternalError;
    if ((values && cudaMemcpy(values + i * nnz, sv, nnz * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (diagonal && cudaMemcpy(diagonal + i * n, sd, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (rhs && cudaMemcpy(rhs + i * n, sr, n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
      return Status::kInternalError;
  }
  if (cudaMemcpy(invalid.data(), invalid_.get(), sizeof(int32_t) * kp, cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  for (int i = 0; i < items; ++i)
    if (invalid[i])
      return Status::kAssemblyFailed;
  return Status::kOk;
}

Status Plan::PcgSolve(int items, const double *values, int values_per_item, const double *rhs,
                      double tolerance, int max_iterations, double *x, fg_linear_info *info)
{
  if (host_only_)
    return Status::kGpuUnavailable;
  if (items <= 0 || items > kMaxItems || !values || !rhs || !x || !info)
    return Status::kInvalidArgument;
  if (items > chunk_cap_)
    return Status::kUnsupportedFeature;
  timing_ = fg_timing{};
  for (int i = 0; i < items; ++i)
    info[i] = fg_linear_info{ToInt(Status::kInvalidArgument), 0, std::numeric_limits<double>::infinity()};
  if (!(tolerance > 0.0) || !(tolerance < 1.0) || !std::isfinite(tolerance) || max_iterations < 0)
    return Status::kOk;
  const bool shared = values_per_item == 0;
  if (!shared && values_per_item != host_.nnz)
    return Status::kInvalidArgument;
  const int kp = PadItems(items);
  Status s = EnsureWorkspace(kp);
  if (s != Status::kOk)
    return s;
  const size_t n = host_.n, n_pad = host_.n_pad, nnz = host_.nnz;
  const int op_items = shared ? 1 : items;
  if ((s = staging_.upload(values, op_items * nnz)) != Status::kOk)
    return s;
  // Diagonal, inverse (BuildJacobiInverseDiagonal, options.cpp:176-199) and rhs, interleaved.
  const int dk = shared ? 1 : kp;
  std::vector<double> d(n_pad * dk, 1.0), inv(n_pad * dk, 0.0), b(n_pad * kp, 0.0);
  bool usable = true;
  for (int i = 0; i < op_items; ++i)
    for (size_t r = 0; r < n; ++r) {
      const double v = values[i * nnz + host_.diag_slot[r]];
      d[r * dk + i] = v;
      const double iv = 1.0 / v;
      if (!std::isfinite(v) || !(v > 0.0) || !std::isnormal(iv)) {
        usable = false;
        inv[r * dk + i] = 0.0;
      } else {
        inv[r * dk + i] = iv;
      }
    }
  for (int i = 0; i < items; ++i)
    for (size_t r = 0; r < n; ++r)
      b[r * kp + i] = rhs[i * n + r];
  if ((s = diag_.upload(d.data(), d.size())) != Status::kOk ||
      (s = invd_.upload(inv.data(), inv.size())) != Status::kOk ||
      (s = rhs_.upload(b.data(), b.size())) != Status::kOk)
    return s;
  const int vk = shared ? 1 : kp;
  if (LaunchScatterCsr(dev_, vk, op_items, staging_.get(), shared ? 0 : static_cast<int>(nnz), values_.get(), nullptr) != cudaSuccess)
    return Status::kInternalError;
  const uint32_t mask = items >= 32 ? 0xffffffffu : ((1u << items) - 1u);
  if (block_size() && cudaMemset(block_fallbacks_.get(), 0, sizeof(int32_t)) != cudaSuccess)
    return Status::kInternalError;
  if ((s = BuildBlocks(kp, items, !shared, false, nullptr)) != Status::kOk)
    return s;
  s = RunPcg(kp, items, mask, tolerance, max_iterations, vk, shared ? 0 : 1, dk, shared ? 0 : 1,
             usable ? 1 : 0, nullptr, block_size() ? blocks64_.get() : nullptr);
  if (s != Status::kOk)
    return s;
  if (block_size()) {
    int32_t fallbacks = 0;
    if (cudaMemcpy(&fallbacks, block_fallbacks_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return Status::kInternalError;
    timing_.block_fallbacks = fallbacks;
  }
  std::vector<double> xi(n_pad * kp), pinfo(3 * kp);
  int32_t err = 0;
  if (cudaMemcpy(xi.data(), x_.get(), xi.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(pinfo.data(), pcg_info_.get(), sizeof(double) * 3 * kp, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&err, error_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  if (err)
    return Status::kInternalError;
  for (int i = 0; i < items; ++i) {
    info[i].status = static_cast<int32_t>(pinfo[3 * i]);
    info[i].iterations = static_cast<int32_t>(pinfo[3 * i + 1]);
    info[i].residual_l2 = pinfo[3 * i + 2];
    for (size_t r = 0; r < n; ++r)
      x[i * n + r] = xi[r * kp + i];
  }
  return Status::kOk;
}

Status Plan::SolveTangent(const double *base_a, const double *base_currents, int m, const double *directions,
                          const fg_solve_options &o, double *da, double *db1, double *db2, double *dflux,
                          fg_linear_info *info)
{
  if (host_only_)
    return Status::kGpuUnavailable;
  if (m <= 0 || !base_a || !directions || !info || (!base_currents && host_.C > 0))
    return Status::kInvalidArgument;
  const size_t N = host_.N, E = host_.E, C = host_.C;
  for (int i = 0; i < m; ++i)
    info[i] = fg_linear_info{ToInt(Status::kInvalidArgument), 0, std::numeric_limits<double>::infinity()};
  // The reference's argument checks (nonlinear_solver.cu:96-104) fail every direction.
  bool valid = o.linear_relative_tolerance > 0.0 && o.linear_relative_tolerance < 1.0 &&
               std::isfinite(o.linear_relative_tolerance) && o.max_linear_iterations >= 0;
  for (size_t i = 0; valid && i < N; ++i)
    valid = std::isfinite(base_a[i]);
  for (size_t i = 0; valid && i < m * C; ++i)
    valid = std::isfinite(directions[i]);
  if (!valid)
    return Status::kOk;
  timing_ = fg_timing{};
  const int cap = std::min(chunk_cap_, kMaxItems);
  const int kp_max = PadItems(std::min(m, cap));
  Status s = EnsureWorkspace(kp_max);
  if (s != Status::kOk)
    return s;
  if ((s = in_warm_.upload(base_a, N)) != Status::kOk || (s = in_currents_.upload(directions, m * C)) != Status::kOk ||
      (da && (s = out_a_.ensure(m * N)) != Status::kOk) || (db1 && (s = out_b1_.ensure(m * E)) != Status::kOk) ||
      (db2 && (s = out_b2_.ensure(m * E)) != Status::kOk) ||
      (dflux && C > 0 && (s = out_flux_.ensure(m * C)) != Status::kOk))
    return s;
  // The consistent Newton Jacobian at the base field, one operator (item 0 of a kp = 1 layout).
  int32_t invalid = 0;
  if (LaunchInterleave(1, 1, static_cast<int>(N), static_cast<int>(N), in_warm_.get(), state_.get(), nullptr) !=
          cudaSuccess ||
      cudaMemset(invalid_.get(), 0, sizeof(int32_t)) != cudaSuccess ||
      LaunchElementKernel(dev_, 1, state_.get(), 1u, 1u, ev_.get(), er_.get(), invalid_.get(), nullptr) != cudaSuccess ||
      LaunchGatherValues(dev_, 1, ev_.get(), 1u, values_.get(), diag_.get(), invd_.get(), invalid_.get(), nullptr) !=
          cudaSuccess ||
      cudaMemcpy(&invalid, invalid_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  timing_.kernel_launches += 3;
  if (invalid) {
    for (int i = 0; i < m; ++i)
      info[i].status = ToInt(Status::kAssemblyFailed);
    return Status::kOk;
  }
  if (block_size() && cudaMemset(block_fallbacks_.get(), 0, sizeof(int32_t)) != cudaSuccess)
    return Status::kInternalError;
  if ((s = BuildBlocks(1, 1, false, false, nullptr)) != Status::kOk)
    return s;
  for (int first = 0; first < m; first += cap) {
    const int k = std::min(cap, m - first), kp = PadItems(k);
    const uint32_t mask = k >= 32 ? 0xffffffffu : ((1u << k) - 1u);
    if (LaunchTangentRhs(dev_, kp, k, in_currents_.get() + static_cast<size_t>(first) * C, rhs_.get(), nullptr) !=
        cudaSuccess)
      return Status::kInternalError;
    timing_.kernel_launches += 1;
    if ((s = RunPcg(kp, k, mask, o.linear_relative_tolerance, o.max_linear_iterations, 1, 0, 1, 0, 1, nullptr,
                    block_size() ? blocks64_.get() : nullptr)) != Status::kOk)
      return s;
    double pinfo[3 * kMaxItems];
    int32_t err = 0;
    if (cudaMemcpy(pinfo, pcg_info_.get(), sizeof(double) * 3 * kp, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(&err, error_.get(), sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
      return Status::kInternalError;
    if (err)
      return Status::kInternalError;
    if (LaunchDerivativeState(dev_, kp, x_.get(), state_.get(), nullptr) != cudaSuccess ||
        LaunchFinalize(dev_, kp, k, state_.get(), da ? out_a_.get() + static_cast<size_t>(first) * N : nullptr,
                       db1 ? out_b1_.get() + static_cast<size_t>(first) * E : nullptr,
                       db2 ? out_b2_.get() + static_cast<size_t>(first) * E : nullptr,
                       dflux && C > 0 ? out_flux_.get() + static_cast<size_t>(first) * C : nullptr,
                       nullptr) != cudaSuccess)
      return Status::kInternalError;
    timing_.kernel_launches += 4;
    for (int i = 0; i < k; ++i) {
      info[first + i].status = static_cast<int32_t>(pinfo[3 * i]);
      info[first + i].iterations = static_cast<int32_t>(pinfo[3 * i + 1]);
      info[first + i].residual_l2 = pinfo[3 * i + 2];
    }
  }
  if ((da && cudaMemcpy(da, out_a_.get(), m * N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (db1 && cudaMemcpy(db1, out_b1_.get(), m * E * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (db2 && cudaMemcpy(db2, out_b2_.get(), m * E * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (dflux && C > 0 && cudaMemcpy(dflux, out_flux_.get(), m * C * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess))
    return Status::kInternalError;
  // A derivative whose B or flux is not finite fails like FinalizeResult's check.
  if (dflux)
    for (int i = 0; i < m; ++i)
      for (size_t c = 0; c < C; ++c)
        if (info[i].status == 0 && !std::isfinite(dflux[i * C + c]))
          info[i].status = ToInt(Status::kNumericalNonfinite);
  return Status::kOk;
}

} // namespace fg
