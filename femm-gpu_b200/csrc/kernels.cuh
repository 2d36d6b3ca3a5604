// kernels.cuh -- device views of the plan and batch workspace, and kernel launchers.
//
// Batch layout: a batch of k items is padded to KP = next power of two (<= 32) and
// every per-row / per-node / per-element / per-position array is item-interleaved:
// element [i][item] lives at i * KP + item.  A warp covers 32 / KP rows x KP items,
// so every SELL-32 column load of a warp touches 32 consecutive doubles.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace fg
{

constexpr int kMaxItems = 32;
// Entries per chunk of the PCG's value ring (per warp: 2 stages x kRingEntries entries x 32
// lanes x 16 bytes of dynamic shared memory).
constexpr int kRingEntries = 4;

struct DevicePlan {
  int32_t N, E, n, n_pad, slices, C, problem_type;
  int64_t nnz, positions;
  const int32_t *row_offsets, *columns, *row_len, *slice_off, *sell_col;
  const int32_t *contrib_off, *contrib, *rhs_off, *rhs_contrib;
  const double *pm_rhs, *circuit_rhs;
  const double *age_val, *age_rhs; // air-gap stiffness [nnz] and load [n]; null without
  const int32_t *elem_nodes, *elem_mat;
  const double *elem_geo;
  const double *mat_nu0, *mat_alpha, *mat_cold, *mat_jpa;
  const int32_t *mat_curve_off, *mat_curve_cnt, *mat_circuit;
  const double *curve_b, *curve_h, *curve_slope;
  const int32_t *node_to_free;
  const int32_t *free_roots; // [n] root node of each free row
  const int8_t *node_sign;
  const double *boundary;
  const int32_t *circuit_elem_off, *circuit_elems;
  double depth_m;
};

// Per-item scalar arguments small enough to pass by value.
struct ItemScalars {
  double v[kMaxItems];
};

// One PCG launch over a batch (shared SELL pattern, per-item or shared operator).
struct PcgArgs {
  int32_t n, n_pad, slices, kp, items;
  const int32_t *slice_off, *row_len, *sell_col;
  // Storage type of values, diagonal, inverse diagonal and every vector: FP64
  // (precision 0) or FP32 (precision 1: SpMV accumulated in FP32, dot products in FP64).
  int32_t precision;
  const void *values;    // [positions][vs]
  int32_t value_stride;  // KP (per-item operators) or 1 (one shared operator)
  int32_t value_item;    // 1 or 0
  const void *diag, *invd; // [n_pad][ds]
  int32_t diag_stride, diag_item;
  int32_t use_inverse;
  // Block-Jacobi (block_size 8 or 32; 0 = Jacobi): inverses in T, entry (i, j) of block
  // b at [(b * bs + j) * bs + i] * block_stride (+ item when block_item), NaN first entry
  // = unusable block.
  const void *blocks;
  int32_t block_size, block_stride, block_item;
  const void *b;
  void *x, *r, *z, *p0, *p1, *q;
  double *partials;   // [2][64][grid]
  unsigned int *barrier;
  int32_t *error;
  double *info;       // [items][3]: status, iterations, residual
  double tolerance;
  const double *item_tolerance; // optional per-item tolerance [items], overrides tolerance
  int32_t max_iterations;
  // 0: verify the true residual at the threshold (the reference's rule).  1: accept on
  // the recursive residual (inner solves whose caller checks the true residual).
  int32_t skip_verification;
  uint32_t active_mask;
  long long timeout_ns;
  // Reliable updates (FP32 storage only): values64 / b64 are the FP64 operator (same
  // layout and strides as values) and right-hand side; the solution accumulates in x64 and
  // is returned there (scaled back); the residual is replaced by the FP64 true residual
  // whenever the recursive residual falls below reliable_delta times its largest value
  // since the previous replacement, and acceptance is the FP64 true-residual rule.
  int32_t reliable;
  double reliable_delta;
  const double *values64, *b64;
  double *x64;
  // Column-index cache (opt-in, FG_PCG_COL_CACHE=1): host copy of slice_off (read by
  // LaunchPcg only, never by the kernel) lets the launch size a shared-memory copy of each
  // CTA's SELL column indices, loaded once per launch; col_cache / col_cache_offset are
  // set by LaunchPcg.
  const int32_t *host_slice_off;
  int32_t col_cache, col_cache_offset;
  // Value ring: the SpMV's operator values staged into shared memory by cp.async one chunk
  // ahead of their use (set by LaunchPcg for 16-byte item vectors).
  int32_t value_ring, value_ring_offset;
  // Launch-shape requests of a plan's autotuner for the value ring and the column-index
  // cache: 0 the default (environment), 1 on where the shape and shared memory allow it,
  // 2 off.  Neither changes any arithmetic, so results do not depend on the choice.
  int32_t ring_request, col_cache_request;
  // CTA shape request: 0 the default (FG_PCG_BLOCK=1024 in the environment: 1024 threads,
  // else 512), 1 CTAs of 1024 threads where the launch allows them (FP64 Jacobi, an even
  // number of row groups), 2 CTAs of 512.  Both shapes give the same bits.
  int32_t block_request;
  // One-reduction form (FP64 Jacobi only; pcg1r_kernel.cuh): t0 / t1 are two more
  // vectors of [n_pad][kp] doubles, and partials must hold 2 x 96 x grid doubles.
  int32_t one_reduction;
  void *t0, *t1;
  // Optional phase trace written by CTA 0 (nanoseconds, summed over the launch):
  // [2q] work before reduction q, [2q+1] wait at its grid barrier, [8] final partial
  // sums, [9] reductions.  q: 0 Phase A, 1 Phase B, 2 verification, 3 set-up.
  unsigned long long *trace;
};
constexpr int kPcgTraceSlots = 10;

// Groups of a multi-plan PCG launch (device arrays): args [groups]; per CTA its group;
// per group its first CTA and CTA count.
struct PcgGroups {
  const PcgArgs *args;
  const int32_t *cta_group, *group_first, *group_size;
};

// Launchers (return cudaError_t of the launch).
cudaError_t LaunchElementKernel(const DevicePlan &p, int kp, const double *state,
                                uint32_t newton_mask, uint32_t active_mask, double *elem_vals,
                                double *elem_rhs, int32_t *invalid, cudaStream_t stream);
cudaError_t LaunchGatherValues(const DevicePlan &p, int kp, const double *elem_vals,
                               uint32_t active_mask, double *values, double *diag, double *invd,
                               int32_t *invalid, cudaStream_t stream);
cudaError_t LaunchGatherRhs(const DevicePlan &p, int kp, const double *elem_rhs,
                            const double *currents, const double *hc_scale, uint32_t active_mask,
                            double *rhs, cudaStream_t stream);
// Block-Jacobi inverses of the assembled operators (blocks of bs rows, bs = 8 or 32),
// written in FP64 (out64) or FP32 (out32); per item when value_item, else one shared set.
// *fallbacks counts the blocks marked unusable.
cudaError_t LaunchBlockInverse(const DevicePlan &p, int kp, int items, int bs, const double *values,
                               int value_item, const double *diag, int diag_item, double *out64,
                               float *out32, int32_t *fallbacks, cudaStream_t stream);
// Cooperative persistent PCG; *grid_out receives the number of CTAs used.
cudaError_t LaunchPcg(PcgArgs args, int *grid_out, int *block_out, cudaStream_t stream);
int PcgMaxGrid(int kp);
// Bound of every grid-wide wait of the PCG launches of plans, fg_csr_pcg and multi-plan
// solves, in nanoseconds (fg_set_wait_limit_ns; default kDefaultWaitLimitNs).
constexpr long long kDefaultWaitLimitNs = 5000000000LL;
long long PcgWaitLimitNs();
long long SetPcgWaitLimitNs(long long ns);
// One cooperative launch of `ctas` CTAs solving every group of t (FP64 Jacobi; every group
// holds kp items: 1, or 32 for the chunks of a wide shared-geometry batch).  The caller
// zeroes the groups' barrier counters and error flags and, when MultiPcgRingBytes(kp) is not
// zero, sets each group's value_ring (offset 0).
cudaError_t LaunchMultiPcg(PcgGroups t, int kp, int ctas, cudaStream_t stream);
// Co-resident CTAs of the multi-plan kernel for kp items per group (its grid limit), 0
// without a device or for an unsupported kp.
int MultiPcgMaxGrid(int kp = 1);
// Dynamic shared memory of the multi-plan kernel's value ring for kp items per group (0:
// no ring for this width).
size_t MultiPcgRingBytes(int kp);
// Whether a PCG kernel exists for this shape (block size 32 in FP64 stops at 16 items).
bool PcgSupported(int kp, int precision, int block_size);
// Doubles of the partials buffer a launch of up to `grid` CTAs needs (the one-reduction
// form reduces three sums per item).
size_t PcgPartialsDoubles(int grid, bool one_reduction);

cudaError_t LaunchNewtonNorms(const DevicePlan &p, int kp, const double *x, const double *state,
                              double *partials, double *norms, cudaStream_t stream);
cudaError_t LaunchNewtonUpdate(const DevicePlan &p, int kp, const double *x, double *state,
                               ItemScalars relax, uint32_t update_mask, cudaStream_t stream);
// State = zero start (fixed values), or warm_item_major for items in warm_mask.
cudaError_t LaunchInitState(const DevicePlan &p, int kp, const double *warm_item_major,
                            int items, uint32_t warm_mask, double *state, cudaStream_t stream);
// Recovery: Armijo trial points, masked state copies and masked resets to the zero start
// (items in mask only; nodal state arrays [N][kp]).
cudaError_t LaunchTrial(const DevicePlan &p, int kp, const double *x, const double *saved,
                        double *state, ItemScalars alpha, uint32_t mask, cudaStream_t stream);
cudaError_t LaunchMaskedCopy(const DevicePlan &p, int kp, uint32_t mask, const double *from, double *to,
                             cudaStream_t stream);
cudaError_t LaunchResetState(const DevicePlan &p, int kp, uint32_t mask, double *state, cudaStream_t stream);
// x[row][kp] = state[root node of row][kp] (free-row form of a nodal state; padding 0).
cudaError_t LaunchStateToFree(const DevicePlan &p, int kp, const double *state, double *x,
                              cudaStream_t stream);
// d = rhs - J x (d may be null) and norms[2][kp] = ||rhs - J x||^2, ||rhs||^2, for the
// system J (values), rhs assembled at a state whose free-row form is x.
cudaError_t LaunchEquationResidual(const DevicePlan &p, int kp, const double *values,
                                   const double *rhs, const double *x, double *d,
                                   double *partials, double *norms, cudaStream_t stream);
// x = x0 + (item in mask ? delta : 0) over [n_pad][kp].
cudaError_t LaunchAddCorrection(const DevicePlan &p, int kp, uint32_t mask, const double *x0,
                                const double *delta, double *x, cudaStream_t stream);
// Tangent multi-RHS: circuit-derivative loads [n_pad][kp] and the nodal derivative state.
cudaError_t LaunchTangentRhs(const DevicePlan &p, int kp, int items, const double *directions, double *rhs,
                             cudaStream_t stream);
cudaError_t LaunchDerivativeState(const DevicePlan &p, int kp, const double *x, double *state,
                                  cudaStream_t stream);
cudaError_t LaunchFinalize(const DevicePlan &p, int kp, int items, const double *state,
                           double *a_out, double *b1_out, double *b2_out, double *flux_out,
                           cudaStream_t stream);
// CSR-ordered copies of assembled values / diagonal / rhs for item `item`.
cudaError_t LaunchExtractCsr(const DevicePlan &p, int kp, int item, const double *values,
                             const double *diag, const double *rhs, double *csr_values,
                             double *diag_out, double *rhs_out, cudaStream_t stream);
// Scatter CSR-ordered operator values into the SELL layout (item-major input).
cudaError_t LaunchScatterCsr(const DevicePlan &p, int kp, int items, const double *csr_values,
                             int32_t values_per_item, double *values, cudaStream_t stream);
// Mixed-precision form: FP32 copies of the assembled operator values, diagonal and
// inverse diagonal.
cudaError_t LaunchToSingle(const DevicePlan &p, int kp, uint32_t mask, const double *val64,
                           const double *diag64, float *val32, float *diag32, float *invd32,
                           cudaStream_t stream);
// Interleave item-major vectors [items][len] into [len_pad][kp] and back.
cudaError_t LaunchInterleave(int kp, int items, int len, int len_pad, const double *in, double *out,
                             cudaStream_t stream);
cudaError_t LaunchDeinterleave(int kp, int items, int len, const double *in, double *out,
                               cudaStream_t stream);

} // namespace fg
