/*
 * femm_gpu.h -- C ABI of libfemmgpu, the B200 (sm_100a) nonlinear magnetostatic solver.
 *
 * The library replaces FEMM-GPU's in-process solver seam for the nonlinear DC
 * magnetostatic path: P1 Newton assembly with B-H reluctivity, permanent-magnet
 * and series-circuit loads, signed periodic/anti-periodic folding, the batched
 * deterministic PCG, and B / flux-linkage recovery.  Plain pointers and sizes
 * only; every call returns a status code with the numbering of the reference's
 * gpu_femm::Status (gpu_solver/src/core/types.h:11-28).  Errors never cross the
 * boundary as exceptions; a failing batch item never poisons the others.
 *
 * Threading: one thread owns a plan; calls are synchronous on return unless the
 * name ends in _device, in which case work is ordered on the given CUDA stream.
 */
#ifndef FEMM_GPU_H
#define FEMM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FG_ABI_VERSION 2

/* Status codes (gpu_solver/src/core/types.h:11-28). */
enum {
  FG_OK = 0,
  FG_INPUT_IO = 1,
  FG_INVALID_ARGUMENT = 2,
  FG_UNSUPPORTED_FEATURE = 3,
  FG_MESH_INVALID = 4,
  FG_BOUNDARY_INVALID = 5,
  FG_GPU_UNAVAILABLE = 6,
  FG_GPU_ALLOCATION_FAILED = 7,
  FG_ASSEMBLY_FAILED = 8,
  FG_LINEAR_SOLVE_NOT_CONVERGED = 9,
  FG_LINEAR_SOLVE_BREAKDOWN = 10,
  FG_NUMERICAL_NONFINITE = 11,
  FG_OUTPUT_IO = 12,
  FG_INTERNAL_ERROR = 13,
  FG_NONLINEAR_SOLVE_NOT_CONVERGED = 14,
  FG_INVALID_MATERIAL = 15
};

enum { FG_PLANAR = 0, FG_AXISYMMETRIC = 1 };
enum { FG_PRECOND_JACOBI = 0, FG_PRECOND_BLOCK_JACOBI = 1 };
enum { FG_PRECISION_FP64 = 0, FG_PRECISION_MIXED = 1 };

/* One material label (gpu_solver/src/physics/nonlinear_model.h:38-51). */
typedef struct fg_material {
  double reluctivity_zero_m_per_h; /* nu0 = 1 / (mu0 mu_r) */
  double alpha_per_t2;             /* nu = nu0 (1 + alpha |B|^2) when no B-H curve */
  double source_j_per_a;           /* coil current density per circuit amp, A/m^2 */
  double h_c_a_per_m;              /* permanent-magnet coercivity */
  double magnetization_deg;        /* permanent-magnet direction */
  int32_t bh_curve_index;          /* -1: no B-H curve */
  int32_t circuit_index;           /* -1: not driven */
  int32_t group_number;
  int32_t reserved;
} fg_material;

/* Raw B-H points, origin first; the library builds FEMM's DC spline from them
 * (gpu_solver/src/physics/nonlinear_model.cpp:13-113). */
typedef struct fg_bh_curve {
  int32_t count;
  const double *b_t;
  const double *h_a_per_m;
} fg_bh_curve;

/* FEMM's native air-gap element (AirGapElement, gpu_solver/src/physics/nonlinear_model.h:
 * 63-81): an annular air band ri < r < ro that is not triangulated.  The band is split
 * into point_count - 1 equal arcs over arc_length_deg; each point carries four (node,
 * weight) pairs -- n0 / n1 the inner-ring nodes that bracket it, n2 / n3 the outer-ring
 * ones, each weight the +1 / -1 sign of the ring copy the node comes from.  inner_shift /
 * outer_shift place the first ring node of each side, in units of one arc.  The band adds
 * a fixed linear stiffness (planar models only). */
typedef struct fg_air_gap_element {
  int32_t antiperiodic;     /* 0 periodic, 1 anti-periodic closure of the band */
  int32_t point_count;      /* arcs + 1, at least 3 */
  double center_x_m, center_y_m;
  double inner_radius_m, outer_radius_m;
  double arc_length_deg;    /* angle the band spans */
  double inner_shift, outer_shift;
  const int32_t *nodes;     /* [4 * point_count]: n0, n1, n2, n3 per point */
  const double *weights;    /* [4 * point_count]: w0, w1, w2, w3 per point */
} fg_air_gap_element;

/* The model (NonlinearModel, gpu_solver/src/physics/nonlinear_model.h:83-100). */
typedef struct fg_model {
  int32_t problem_type; /* FG_PLANAR or FG_AXISYMMETRIC (x = r, y = z) */
  int32_t node_count;
  const double *node_xy; /* [2 * node_count] metres, interleaved */
  int32_t triangle_count;
  const int32_t *triangle_nodes;    /* [3 * triangle_count], counter-clockwise */
  const int32_t *triangle_material; /* [triangle_count] */
  int32_t material_count;
  const fg_material *materials;
  int32_t curve_count;
  const fg_bh_curve *curves;
  int32_t dirichlet_count;
  const int32_t *dirichlet_nodes;
  const double *dirichlet_values;
  int32_t constraint_count;
  const int32_t *constraint_nodes; /* [2 * constraint_count]: A(b) = sign * A(a) */
  const int8_t *constraint_signs;  /* [constraint_count], +1 periodic / -1 anti-periodic */
  int32_t circuit_count;
  double depth_m;
  /* Appended in ABI version 2; zero them (or zero-initialise the struct) for none. */
  int32_t air_gap_count;
  const fg_air_gap_element *air_gap_elements;
} fg_model;

typedef struct fg_plan_options {
  /* FG_PRECOND_JACOBI (the reference default) or FG_PRECOND_BLOCK_JACOBI: dense inverses
   * of contiguous block_size-row principal blocks (the reference's opt-in
   * `--preconditioner block-jacobi`, gpu_solver/src/app/cli.cpp:39-46, block_size 8).
   * block_size 32 runs at most 16 items per launch (fg_pcg_solve: items <= 16). */
  int32_t preconditioner;
  int32_t block_size;     /* block-Jacobi rows per block: 8 or 32 */
  int32_t precision;      /* FG_PRECISION_*: mixed = FP32 inner PCG in FP64 defect correction */
  int32_t flags;          /* FG_PLAN_HOST_ONLY: build and validate the host topology only */
} fg_plan_options;

/* fg_plan_options.flags: a host-only plan needs no GPU; it answers the topology and
 * introspection calls, and every device call on it returns FG_GPU_UNAVAILABLE. */
/* FG_PLAN_PCG_FROM_ITERATE (no counterpart in the reference, whose inner PCG starts every
 * Newton solve from x = 0): the inner PCG solves for the correction from the current
 * Newton iterate, J delta = rhs - J x0, to ||rhs - J (x0 + delta)|| <= tol ||rhs|| -- the
 * same acceptance rule from a better starting point, so a good iterate or warm start
 * costs fewer PCG iterations. */
/* FG_PLAN_PCG_ONE_REDUCTION (no counterpart in the reference; FP64 Jacobi plans only):
 * the inner PCG runs Chronopoulos and Gear's one-reduction rearrangement of CG -- one
 * grid-wide synchronisation per iteration instead of two, at the price of three gathered
 * vectors per SpMV entry instead of two and two more workspace vectors.  It pays where a
 * CG iteration is short (meshes of tens of thousands of rows).  Acceptance is unchanged
 * (the true-residual check); results agree with the default form within the solve's
 * tolerance, not bit for bit.  With block-Jacobi or mixed precision fg_plan_create
 * returns FG_UNSUPPORTED_FEATURE. */
enum { FG_PLAN_HOST_ONLY = 1, FG_PLAN_PCG_FROM_ITERATE = 2, FG_PLAN_PCG_ONE_REDUCTION = 4 };

/* NonlinearOptions (gpu_solver/src/physics/nonlinear_model.h:102-109). */
typedef struct fg_solve_options {
  double relative_tolerance;
  int32_t max_newton_iterations;
  int32_t max_linear_iterations;
  double linear_relative_tolerance;
  int32_t recover_nonconvergence;
  int32_t adaptive_linear_tolerance;
} fg_solve_options;

/* Per-item result summary (NonlinearSolveResult fields, nonlinear_model.h:132-145). */
typedef struct fg_item_info {
  int32_t status;
  int32_t iterations;  /* Newton iterations */
  double residual_l2;  /* last relative Newton step */
  int32_t linear_iterations;
  /* 0 zero start; 1 started from the supplied warm start; 2 warm start supplied but
   * rejected by the learned-warm-start guard (its equation residual was not below the
   * zero start's), zero start used. */
  int32_t warm_start;
  double last_linear_tolerance;
  double verified_equation_residual_relative;
} fg_item_info;

/* SolveInfo of one linear solve (gpu_solver/src/core/types.h:51-55). */
typedef struct fg_linear_info {
  int32_t status;
  int32_t iterations;
  double residual_l2;
} fg_linear_info;

typedef struct fg_plan_sizes {
  int64_t node_count;
  int64_t triangle_count;
  int64_t rows;  /* free rows after signed folding */
  int64_t nnz;   /* symbolic CSR entries */
  int32_t circuit_count;
  int32_t problem_type;
  int64_t device_bytes; /* device memory currently held by the plan */
  int64_t matrix_contributors; /* element terms summed into CSR slots */
  int64_t rhs_contributors;    /* element terms summed into free rows */
} fg_plan_sizes;

typedef struct fg_timing {
  double assembly_ms;
  double pcg_ms;
  double update_ms;
  double finalize_ms;
  int64_t newton_iterations;
  int64_t pcg_iterations;   /* summed over the PCG launches (max over items per launch) */
  int64_t kernel_launches;  /* of this library's kernels */
  int64_t pcg_launches;
  int32_t pcg_grid;         /* cooperative CTAs of the last PCG launch */
  int32_t pcg_block;
  /* Phase trace of PCG CTA 0, filled only when the environment variable FG_PCG_TRACE=1
   * is set when the plan is created: milliseconds of [0] SpMV phase work, [1] its grid
   * wait, [2] update phase work, [3] its wait, [4] true-residual work, [5] its wait,
   * [6] set-up work, [7] its wait, [8] final partial sums; [9] number of reductions. */
  double pcg_phase_ms[10];
  int64_t mixed_fallbacks; /* mixed form: item solves redone by the FP64 PCG */
  int64_t block_inverses;  /* block-Jacobi: blocks factored (summed over builds) */
  int64_t block_fallbacks; /* block-Jacobi: blocks found unusable (diagonal used instead) */
} fg_timing;

typedef struct fg_plan fg_plan;

/* Reference production options: ProductionSampleOptions
 * (gpu_solver/src/physics/nonlinear_model.cpp:195-205). */
void fg_production_options(fg_solve_options *options);

const char *fg_status_name(int status);
int fg_abi_version(void);

/* Bound, in nanoseconds, of every grid-wide wait inside the PCG launches of plans,
 * fg_csr_pcg and multi-plan solves (default 5 s; ns <= 0 restores the default); returns
 * the previous bound.  When a wait runs out, every CTA of the launch returns and the call
 * reports FG_INTERNAL_ERROR; the CUDA context stays usable.  The reference bounds its
 * device loops the same way (gpu_solver/src/solvers/pcg_kernels.cu:555-566); this setter
 * is the test hook that makes such a wait run out. */
int64_t fg_set_wait_limit_ns(int64_t ns);

/* NonlinearP1Solver::Initialize + device plan set-up (nonlinear_solver.cu:784-800,
 * nonlinear_assembly.cu:362-441, nonlinear_topology.cpp:12-248). */
int fg_plan_create(const fg_model *model, const fg_plan_options *options, fg_plan **plan);
void fg_plan_destroy(fg_plan *plan);
int fg_plan_sizes_get(const fg_plan *plan, fg_plan_sizes *sizes);

/* Symbolic CSR and signed maps (Assembly fields row_offsets, column_indices,
 * node_to_free, node_sign, boundary_values; linear_model.h:9-23).  Any pointer may be NULL. */
int fg_plan_symbolic(const fg_plan *plan, int32_t *row_offsets, int32_t *columns,
                     int32_t *node_to_free, int8_t *node_sign, double *boundary_values);

/* Gather plan of the device assembly (the per-slot / per-row contributor lists of
 * PreparedNonlinearAssembly, nonlinear_topology.cpp:87-179 and :234-248), in
 * element order.  slot_offsets [nnz + 1]; slot_entries [3 * matrix_contributors] as
 * (triangle, symmetric local pair 0..5 = 00,01,02,11,12,22, sign);
 * row_offsets [rows + 1]; row_entries [3 * rhs_contributors] as (triangle, local row, sign);
 * pm_rhs [rows]; circuit_rhs [circuits * rows].  Any pointer may be NULL. */
int fg_plan_contributors(const fg_plan *plan, int32_t *slot_offsets, int32_t *slot_entries,
                         int32_t *row_offsets, int32_t *row_entries, double *pm_rhs,
                         double *circuit_rhs);

/* The fixed air-gap element terms of the plan (PreparedNonlinearAssembly::age_values /
 * age_rhs, nonlinear_topology.cpp:180-262): values [nnz] the band stiffness per CSR slot,
 * rhs [rows] the load that fixed ring nodes put on free rows.  Zeros when the model has no
 * air-gap element.  Either pointer may be NULL. */
int fg_plan_air_gap(const fg_plan *plan, double *values, double *rhs);

/* Device Newton assembly at given nodal states (DeviceNonlinearAssemblyPlan::Assemble,
 * nonlinear_assembly.cu:229-309).  states [items * N]; currents [items * C];
 * use_newton [items]; outputs in CSR order: values [items * nnz], diagonal and
 * rhs [items * rows].  Any output may be NULL. */
int fg_assemble(fg_plan *plan, int32_t items, const double *states, const double *currents,
                const int32_t *use_newton, double *values, double *diagonal, double *rhs);

/* Deterministic Jacobi PCG on the plan's CSR pattern (GpuCsrSolver batch modes,
 * csr_solver.cu:204-503).  values [items * nnz] CSR order (values_per_item = 0
 * shares one operator), rhs [items * rows] -> x [items * rows]. */
int fg_pcg_solve(fg_plan *plan, int32_t items, const double *values, int32_t values_per_item,
                 const double *rhs, double relative_tolerance, int32_t max_iterations, double *x,
                 fg_linear_info *info);

/* Generic CSR PCG on an arbitrary SPD system (GpuCsrSolver::Initialize + Solve /
 * SolveBatch / SolveCurrentOperatorBatch, csr_solver.cu:25-390). */
int fg_csr_pcg(int32_t n, const int32_t *row_offsets, const int32_t *columns,
               const double *values, int32_t values_per_item, const double *diagonal,
               int32_t items, const double *rhs, double relative_tolerance,
               int32_t max_iterations, double *x, fg_linear_info *info);

/* The same deterministic PCG on one CSR system with no memory allocation at all.  This
 * entry point has no counterpart in the reference.  It is for callers that may not
 * allocate GPU memory when they solve -- code running inside a memory pool that owns the
 * device, real-time loops that forbid allocator calls, plug-in hosts that only lend their
 * own buffers.  Every array argument is DEVICE memory owned by the caller (row_offsets
 * [n + 1], columns / values [row_offsets[n]], diagonal / rhs / x [n]); info is host
 * memory; work is ordered on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * the call returns when x and info are final: it synchronises `stream`, reading a small
 * status block back to the host.  x is written only by a solve that ran to its end; when
 * the call returns FG_INTERNAL_ERROR, info->status says so and x is left as it was.  All other memory is one fixed file-scope
 * device array (about 5.5 MB per device that loads the library, held until exit), so no
 * cudaMalloc, cudaFree or allocating library routine is called.
 * Limits: n <= FG_NOALLOC_MAX_ROWS and at most FG_NOALLOC_MAX_POSITIONS SELL-32 slots
 * (entries after padding each 32-row slice to its longest row); larger systems, bad
 * offsets or columns and non-finite entries return FG_INVALID_ARGUMENT.
 * Every call on a device shares that array and overwrites it: calls that overlap on the
 * GPU race and must be serialised by the caller.  The first call on each device, with
 * that device current, looks up the array's device address; make it before any stream
 * capture begins. */
#define FG_NOALLOC_MAX_ROWS 16384
#define FG_NOALLOC_MAX_POSITIONS 262144
int fg_csr_pcg_noalloc(int32_t n, const int32_t *row_offsets, const int32_t *columns,
                       const double *values, const double *diagonal, const double *rhs,
                       double relative_tolerance, int32_t max_iterations, double *x,
                       fg_linear_info *info, void *stream);

/* Batched nonlinear solve (NonlinearP1Solver::SolveBatch, nonlinear_solver.cu:183-530;
 * warm starts as in Solve, :686-698).  Host buffers:
 *   currents [items * C]; hc_scale [items] or NULL (per-item permanent-magnet
 *   coercivity scale); warm_a [items * N] or NULL;
 *   a_out [items * N], b1_out / b2_out [items * E] (Bx/By or Br/Bz), flux_out [items * C],
 *   info [items].  Output pointers may be NULL. */
int fg_solve_batch(fg_plan *plan, int32_t items, const double *currents, const double *hc_scale,
                   const double *warm_a, const fg_solve_options *options, double *a_out,
                   double *b1_out, double *b2_out, double *flux_out, fg_item_info *info);

/* Same, with every array a device pointer and work ordered on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  info stays a host pointer. */
int fg_solve_batch_device(fg_plan *plan, int32_t items, const double *currents,
                          const double *hc_scale, const double *warm_a,
                          const fg_solve_options *options, double *a_out, double *b1_out,
                          double *b2_out, double *flux_out, fg_item_info *info, void *stream);

/* First-order response about a converged operating point (SolveTangentMultiRhs,
 * gpu_solver/src/solvers/nonlinear_solver.cu:85-172): the consistent Newton Jacobian J is
 * assembled once at base_a [node_count] (base_currents [circuit_count] name the operating
 * point), and J dA_i = S_i is solved for every direction i -- S_i = sum over circuits of
 * directions[i][c] times the circuit's per-amp source load, no magnet or boundary terms --
 * in shared-operator PCG launches of up to 32 directions (16 with 32-row blocks), at
 * options->linear_relative_tolerance within options->max_linear_iterations.  Outputs are host
 * arrays and may be NULL: da [m][node_count] (zero on fixed nodes), db1 / db2
 * [m][triangle_count], dflux [m][circuit_count] (the differential inductances for unit
 * directions).  info[i] carries each direction's PCG status, iterations and residual;
 * invalid arguments (non-finite base or directions, a bad tolerance) set every info[i] to
 * FG_INVALID_ARGUMENT as the reference does. */
int fg_solve_tangent(fg_plan *plan, const double *base_a, const double *base_currents, int32_t directions,
                     const double *direction_currents, const fg_solve_options *options, double *da,
                     double *db1, double *db2, double *dflux, fg_linear_info *info);

/* Gives a host-only plan (FG_PLAN_HOST_ONLY) its device side -- the uploads and set-up
 * fg_plan_create does for a device plan -- so that the host preparation (validation,
 * splines, signed folding, symbolic CSR, gather plan) can run on another thread, ahead of
 * the GPU work.  FG_OK on a plan that already has it; FG_GPU_UNAVAILABLE without a GPU. */
int fg_plan_attach_device(fg_plan *plan);

/* Timing and launch counters of the last solve on this plan. */
int fg_plan_last_timing(const fg_plan *plan, fg_timing *timing);

/* The plan's PCG launch shapes.  At the first PCG launch of each (items per launch,
 * precision, block size) a plan times its candidate shapes -- the operator-value ring in
 * shared memory on / off, the per-CTA column-index cache off / on -- on the system it is
 * about to solve (a short run of the same kernel), and keeps the fastest for every later
 * launch of that key.  Neither knob changes any arithmetic: results are the same bits
 * whatever the choice.  No counterpart in the reference (its kernel shape is fixed,
 * gpu_solver/src/solvers/options.cpp:43-53).  FG_PCG_TUNE=0 in the environment keeps the
 * defaults.  Writes at most `capacity` entries; returns the number of tuned keys. */
typedef struct fg_pcg_shape {
  int32_t items;        /* items per launch (the padded batch width) */
  int32_t precision;    /* FG_PRECISION_FP64 or FG_PRECISION_MIXED (the inner FP32 launch) */
  int32_t block_size;   /* 0 Jacobi, 8 or 32 block-Jacobi */
  int32_t value_ring;   /* 1 chosen on, 0 off */
  int32_t column_cache; /* 1 chosen on, 0 off */
  int32_t candidates;   /* shapes timed (those the kernel shape admits) */
  /* per candidate: [0..3] 512-thread CTAs, ring on / off x cache off / on; [4] 1024-thread
   * CTAs (two row groups each, FP64 Jacobi with an even number of row groups), ring on,
   * cache off; 0 if not timed */
  double us_per_iteration[5];
  int32_t threads_per_block; /* the chosen CTA shape: 512 or 1024 (the same bits either way) */
  int32_t reserved;
} fg_pcg_shape;
int fg_plan_pcg_shapes(const fg_plan *plan, int32_t capacity, fg_pcg_shape *shapes);

/* FEMM DC B-H spline and evaluation (nonlinear_model.cpp:13-148): host functions
 * exposed for parity checks.  b/h are smoothed in place; slope [count]. */
int fg_bh_build(int32_t count, double *b, double *h, double *slope, double *cold_secant,
                int32_t *smoothing_passes);
void fg_bh_eval(int32_t count, const double *b, const double *h, const double *slope,
                double field_b, double *h_dh_nu_dnu);

/* ------------------------------------------------------------------------------------
 * Heterogeneous batches (no counterpart in the reference, which solves one operator per
 * launch group).  Independent meshes -- one plan each, of any size -- are solved in
 * lock-step, one sample per plan: per Newton iteration every active plan is assembled and
 * all their PCG solves run in ONE cooperative launch, each on its own group of CTAs, with
 * per-plan convergence; from the second iteration the assembly + PCG + norm sequence is a
 * replayed CUDA graph.  An online tuner divides the CTAs by predicted cost (rows x
 * iterations, from each plan's previous Newton step).  Plans must use the FP64 Jacobi
 * form without FG_PLAN_PCG_FROM_ITERATE or FG_PLAN_PCG_ONE_REDUCTION (FG_UNSUPPORTED_FEATURE
 * otherwise); they are borrowed and must outlive the fg_multi.
 * ------------------------------------------------------------------------------------ */
typedef struct fg_multi fg_multi;

typedef struct fg_multi_timing {
  double total_ms;          /* wall time of the last fg_multi_solve */
  int64_t newton_steps;     /* lock-step Newton iterations */
  int64_t pcg_launches;     /* multi-plan PCG launches */
  int64_t graph_launches;   /* replays of captured iterations */
  int64_t graph_captures;   /* (re)captures: once per distinct set of active plans */
  int64_t kernel_launches;  /* launches outside graphs, plus captured kernels per replay */
  int32_t max_ctas;         /* largest CTA count of one PCG launch */
  int32_t reserved;
} fg_multi_timing;

int fg_multi_create(fg_plan *const *plans, int32_t count, fg_multi **multi);
void fg_multi_destroy(fg_multi *multi);
/* One sample per plan: currents[m] -> [C_m]; outputs per plan (host, each may be NULL):
 * a_out[m] [N_m], b1_out[m] / b2_out[m] [E_m], flux_out[m] [C_m]; info [count]. */
int fg_multi_solve(fg_multi *multi, const double *const *currents, const fg_solve_options *options,
                   double *const *a_out, double *const *b1_out, double *const *b2_out,
                   double *const *flux_out, fg_item_info *info);
int fg_multi_last_timing(const fg_multi *multi, fg_multi_timing *timing);

/* ------------------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference).  A reduced basis of A (mean +
 * rank orthonormal modes) whose coefficients a small MLP predicts from per-sample
 * features (circuit currents and magnet-angle terms, normalised by the caller's shift and
 * scale).  The network is trained and evaluated by this library's own kernels in FP32;
 * the basis and the warm start are FP64.  The Newton solve starts from the prediction only
 * where its equation residual ||K(A) A - b|| is below the zero start's, and always finishes
 * at the unchanged tolerances.
 * ------------------------------------------------------------------------------------ */
typedef struct fg_mlp fg_mlp;
typedef struct fg_warm fg_warm;

/* MLP inputs -> hidden -> hidden -> outputs, exact-erf GELU after each hidden layer,
 * seeded uniform(+-1/sqrt(fan_in)) initialisation.  Parameter vector layout (FP32):
 * W1[hidden][inputs], b1[hidden], W2[hidden][hidden], b2[hidden], W3[outputs][hidden],
 * b3[outputs]. */
int fg_mlp_create(int32_t inputs, int32_t hidden, int32_t outputs, uint64_t seed, fg_mlp **mlp);
void fg_mlp_destroy(fg_mlp *mlp);
int64_t fg_mlp_parameter_count(const fg_mlp *mlp);
int fg_mlp_get_parameters(const fg_mlp *mlp, float *parameters);
int fg_mlp_set_parameters(fg_mlp *mlp, const float *parameters);
/* y [batch][outputs] = f(x [batch][inputs]); host arrays. */
int fg_mlp_forward(fg_mlp *mlp, int32_t batch, const float *x, float *y);
/* loss = 0.5 / batch * sum (f(x) - t)^2 and d loss / d parameters (parameter layout). */
int fg_mlp_loss_gradient(fg_mlp *mlp, int32_t batch, const float *x, const float *t, float *loss,
                         float *gradient);
/* Adam (beta 0.9 / 0.999, eps 1e-8) over `epochs` seeded shuffles of (x, t) in minibatches
 * of `batch` rows; *final_loss = the loss over all samples afterwards. */
int fg_mlp_train(fg_mlp *mlp, int32_t samples, const float *x, const float *t, int32_t epochs,
                 int32_t batch, float learning_rate, uint64_t seed, float *final_loss);

/* mean [N] and basis [rank][N] of the plan's nodal A; mlp (borrowed, outputs == rank) may
 * be NULL for a projection-only model.  feature_shift / feature_scale [mlp inputs],
 * coeff_shift / coeff_scale [rank]: coefficients = coeff_shift + coeff_scale * f(x),
 * x = (features - feature_shift) / feature_scale. */
int fg_warm_create(const fg_plan *plan, int32_t rank, const double *mean, const double *basis,
                   fg_mlp *mlp, const float *feature_shift, const float *feature_scale,
                   const double *coeff_shift, const double *coeff_scale, fg_warm **warm);
void fg_warm_destroy(fg_warm *warm);
/* coeffs [k][rank] = basis (a [k][N] - mean); host arrays, or device arrays on `stream`. */
int fg_warm_project(fg_warm *warm, int32_t k, const double *a, double *coeffs);
int fg_warm_project_device(fg_warm *warm, int32_t k, const double *a, double *coeffs, void *stream);
/* Predicted warm starts a [k][N] from features [k][inputs]; host arrays. */
int fg_warm_predict(fg_warm *warm, int32_t k, const float *features, double *a);
/* fg_solve_batch from the learned warm start of each item (features [items][inputs]),
 * guarded as described above; info[i].warm_start tells which start each item used. */
int fg_solve_batch_learned(fg_plan *plan, fg_warm *warm, int32_t items, const double *currents,
                           const double *hc_scale, const float *features,
                           const fg_solve_options *options, double *a_out, double *b1_out,
                           double *b2_out, double *flux_out, fg_item_info *info);

/* ---- Frozen-state postprocessing: weighted-stress force / torque and air-gap B ----
 *
 * ComputeFrozenPostprocess (gpu_solver/src/postprocess/field_postprocess.cpp:341-403) with
 * its reusable FrozenPostprocessPlan (:205-339) and FEMM's weighted-stress mask
 * (weighted_stress.cu:24-193): the mask is the sqrt(area)-weighted Laplace solution, 1 on
 * the selected region, 0 on other non-air regions and on the Dirichlet nodes (symmetry
 * apex nodes excepted), periodic across every node constraint whatever its magnetic sign,
 * solved by the library's PCG on the GPU and thresholded at 0.5.  Planar plans only.
 *
 * Selection: selected_group_number >= 0 selects every label of that FEMM group, else the
 * label index selected_material_label; likewise air. */
typedef struct fg_postprocess_options {
  int32_t selected_material_label; /* 1 */
  int32_t air_material_label;      /* 3 */
  int32_t selected_group_number;   /* -1 */
  int32_t air_group_number;        /* -1 */
  double airgap_radius_m;          /* probes at (r cos t, r sin t); each must fall in air */
  int32_t airgap_angle_count;
  const double *airgap_angles_rad;
  int32_t max_mask_iterations;     /* 256 */
  double mask_relative_tolerance;  /* 1e-12 */
  int32_t symmetry_apex_count;     /* anti-periodic sector apex nodes: magnetic zero only */
  const int32_t *symmetry_apex_nodes;
} fg_postprocess_options;

/* FrozenPostprocessResult minus the samples (written to a separate array). */
typedef struct fg_postprocess_result {
  int32_t status;
  int32_t reserved;
  double force_x_n;
  double force_y_n;
  double torque_nm;
} fg_postprocess_result;

typedef struct fg_postprocess fg_postprocess;

/* The FrozenPostprocessOptions defaults (postprocess.h:20-33). */
void fg_postprocess_default_options(fg_postprocess_options *options);
/* Builds the reusable postprocess (mask, element geometry, probe elements) for the plan's
 * model; mask [node_count] of 0 / 1 values, or NULL to solve it on the GPU.  Returns the
 * plan status (FG_INVALID_MATERIAL for a selection that is absent or touches another
 * non-air region, FG_BOUNDARY_INVALID for contradictory fixed mask values, FG_INVALID_ARGUMENT
 * for bad options or a probe outside air, the mask PCG's status ...); *out is NULL unless
 * FG_OK.  The postprocess copies what it needs and does not borrow the plan. */
int fg_postprocess_create(const fg_plan *plan, const fg_postprocess_options *options,
                          const double *mask, fg_postprocess **out);
void fg_postprocess_destroy(fg_postprocess *postprocess);
int32_t fg_postprocess_probe_count(const fg_postprocess *postprocess);
/* The thresholded mask [node_count]. */
int fg_postprocess_mask(const fg_postprocess *postprocess, double *mask);
/* Force, torque and radial air-gap B of `items` solutions (host arrays, item-major:
 * a [items][node_count], b1 / b2 [items][triangle_count]); results [items],
 * airgap_radial_b_t [items][probe_count] (may be NULL when there are no probes).
 * Per-item failures (FG_NUMERICAL_NONFINITE, FG_MESH_INVALID) are in results[i].status. */
int fg_postprocess_compute(const fg_postprocess *postprocess, int32_t items, const double *a,
                           const double *b1, const double *b2, fg_postprocess_result *results,
                           double *airgap_radial_b_t);
/* The same from DEVICE solutions (item-major, as above) on `stream` (a cudaStream_t): one
 * deterministic reduction kernel for force and torque over all items, and a gather of
 * the few values each probe's smoothing reads; results stay host memory. */
int fg_postprocess_compute_device(fg_postprocess *postprocess, int32_t items,
                                  const double *a, const double *b1, const double *b2,
                                  fg_postprocess_result *results, double *airgap_radial_b_t,
                                  void *stream);
/* Force / torque / air-gap derivatives of `directions` tangent solutions about the base
 * field (ComputeFrozenTangentPostprocess, field_postprocess.cpp:405-520): the bilinear cross
 * term of the weighted-stress density between base B (base_b1 / base_b2 [triangle_count])
 * and each dB, and the smoothed radial dB at the probes.  da [m][node_count], db1 / db2
 * [m][triangle_count]; results [m] (N/A, N m/A), airgap_radial_b_t [m][probe_count] (T/A). */
int fg_postprocess_tangent(const fg_postprocess *postprocess, int32_t directions, const double *base_b1,
                           const double *base_b2, const double *da, const double *db1, const double *db2,
                           fg_postprocess_result *results, double *airgap_radial_b_t);
/* One-shot ComputeFrozenPostprocess: create, compute one item, destroy.  A plan failure is
 * returned in result->status (the call itself returns FG_OK). */
int fg_postprocess_frozen(const fg_plan *plan, const fg_postprocess_options *options,
                          const double *a, const double *b1, const double *b2,
                          fg_postprocess_result *result, double *airgap_radial_b_t);

/* The sliding-band postprocess of a plan whose model carries native air-gap elements
 * (ComputeAirGapElementPostprocess, gpu_solver/src/postprocess/airgap_postprocess.cpp:
 * 44-161): B at the centre of every band arc from nodal A, the Maxwell-stress force and
 * torque summed over the arcs of every band, and the radial B of the first band's Fourier
 * series at angles_rad (FEMM's mo_getgapb).  a [items][node_count] (host); results [items];
 * airgap_radial_b_t [items][angle_count].  Per-item statuses as the reference's
 * (FG_INVALID_ARGUMENT without a band or for a non-finite angle, FG_MESH_INVALID for a
 * degenerate band, FG_NUMERICAL_NONFINITE); the call returns FG_OK unless its arguments
 * are unusable. */
int fg_air_gap_postprocess(const fg_plan *plan, int32_t items, const double *a, int32_t angle_count,
                           const double *angles_rad, fg_postprocess_result *results,
                           double *airgap_radial_b_t);
/* Derivatives of the same along tangent solutions da [directions][node_count] about base_a
 * [node_count] (ComputeAirGapElementTangentPostprocess, airgap_postprocess.cpp:163-285):
 * force / torque per amp from the cross terms of B and dB, radial dB from the series of the
 * first band's dBr.  results [directions]; airgap_radial_b_t [directions][angle_count]. */
int fg_air_gap_tangent(const fg_plan *plan, int32_t directions, const double *base_a, const double *da,
                       int32_t angle_count, const double *angles_rad, fg_postprocess_result *results,
                       double *airgap_radial_b_t);

#ifdef __cplusplus
}
#endif
#endif
