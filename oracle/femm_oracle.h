/*
 * femm_oracle.h -- CPU oracle for the nonlinear magnetostatic hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, single-threaded restatement of
 * the reference algorithm (FEMM-GPU gpu_solver) used by tests/, the smoke check
 * and the CPU-baseline leg of bench.py as the checker.  The product library
 * (libfemmgpu) never links, loads or calls it.
 *
 * Parity is pinned against the reference's own golden vectors
 * (tests/fixtures/35PN230_v1 reference_samples.txt / smoothing_reference.txt,
 * the self-test and physics-regression known answers, the stock-FEMM strip and
 * axisymmetric artifacts) and against oracle/_ref, the reference's host
 * sources compiled here.
 */
#ifndef FEMM_ORACLE_H
#define FEMM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: identical numbering to gpu_solver/src/core/types.h:11-28. */
enum {
  OR_OK = 0, OR_INPUT_IO = 1, OR_INVALID_ARGUMENT = 2, OR_UNSUPPORTED = 3, OR_MESH_INVALID = 4,
  OR_BOUNDARY_INVALID = 5, OR_GPU_UNAVAILABLE = 6, OR_GPU_ALLOC = 7, OR_ASSEMBLY_FAILED = 8,
  OR_LINEAR_NOT_CONVERGED = 9, OR_LINEAR_BREAKDOWN = 10, OR_NONFINITE = 11, OR_OUTPUT_IO = 12,
  OR_INTERNAL = 13, OR_NONLINEAR_NOT_CONVERGED = 14, OR_INVALID_MATERIAL = 15
};

/* A B-H curve after the FEMM DC spline build (b/h may have been smoothed). */
typedef struct {
  int32_t count;
  double *b;      /* [count] */
  double *h;      /* [count] */
  double *slope;  /* [count] */
  double cold_secant;
  int32_t smoothing_passes;
} or_curve;

/* A native air-gap element, laid out as fg_air_gap_element.  The restatement does not
 * assemble these (models carrying them are refused with OR_UNSUPPORTED); the
 * reference build (ref_driver.cpp) maps them onto AirGapElement. */
typedef struct {
  int32_t antiperiodic, point_count;
  double center_x_m, center_y_m, inner_radius_m, outer_radius_m, arc_length_deg;
  double inner_shift, outer_shift;
  const int32_t *nodes;  /* [4 * point_count] */
  const double *weights; /* [4 * point_count] */
} or_air_gap;

typedef struct {
  int32_t problem_type; /* 0 planar, 1 axisymmetric (x = r, y = z) */
  int32_t node_count;
  const double *xy; /* [2N] metres */
  int32_t tri_count;
  const int32_t *tri;     /* [3E] */
  const int32_t *tri_mat; /* [E] */
  int32_t mat_count;
  const double *nu0, *alpha, *j_per_a, *hc, *mag_deg; /* [M] each */
  const int32_t *curve_index, *circuit_index;          /* [M] each, -1 = none */
  int32_t curve_count;
  const int32_t *curve_offsets; /* [curve_count + 1] into curve_b/curve_h (raw points) */
  const double *curve_b, *curve_h;
  int32_t dir_count;
  const int32_t *dir_nodes;
  const double *dir_values;
  int32_t con_count;
  const int32_t *con_a, *con_b; /* A(b) = sign * A(a) */
  const int8_t *con_sign;
  int32_t circuit_count;
  double depth_m;
  int32_t age_count;
  const or_air_gap *ages;
} or_model;

typedef struct {
  double relative_tolerance;
  int32_t max_newton_iterations;
  int32_t max_linear_iterations;
  double linear_relative_tolerance;
  int32_t recover_nonconvergence;
  int32_t adaptive_linear_tolerance;
} or_options;

typedef struct {
  int32_t status;
  int32_t iterations;
  double residual_l2;
  int32_t linear_iterations;
  double last_linear_tolerance;
  double verified_equation_residual_relative;
} or_info;

/* FEMM DC natural-cubic B-H spline (nonlinear_model.cpp:13-113).  b and h are
 * modified in place by smoothing; slope must hold count doubles. */
int or_bh_build(int32_t count, double *b, double *h, double *slope, double *cold_secant,
                int32_t *smoothing_passes);
/* H, dH/dB, nu = H/B, dnu/d(B^2) at |field_b| (nonlinear_model.cpp:115-148). out[4]. */
void or_bh_eval(int32_t count, const double *b, const double *h, const double *slope,
                double field_b, double *out);

/* Signed DOF map (signed_node_constraints.h:33-106).  Returns 0 ok, 1 invalid constraint,
 * 2 contradictory cycle, 3 invalid fixed value. */
int or_signed_dofs(int32_t node_count, int32_t con_count, const int32_t *con_a,
                   const int32_t *con_b, const int8_t *con_sign, int32_t dir_count,
                   const int32_t *dir_nodes, const double *dir_values, int32_t *node_root,
                   int8_t *node_sign, int32_t *node_to_free, double *boundary_values,
                   int32_t *free_count);

/* Model validation (nonlinear_model.cpp:223-319, AGE part excluded). */
int or_validate(const or_model *m);

/* Reduced Newton system from the host assembler (nonlinear_model.cpp:453-627 + :321-394). */
typedef struct or_system or_system;
int or_assemble(const or_model *m, const double *a_old, const double *currents, int use_newton,
                or_system **out);
void or_system_free(or_system *s);
int32_t or_system_rows(const or_system *s);
int32_t or_system_nnz(const or_system *s);
/* Any pointer may be NULL. rhs = rhs_per_amp + rhs_offset. */
void or_system_copy(const or_system *s, int32_t *row_offsets, int32_t *columns, double *values,
                    double *diagonal, double *rhs, int32_t *node_to_free, int8_t *node_sign,
                    double *boundary_values, double *circuit_sources /* [c * rows] signed */);

/* Preconditioner used by or_pcg and the Newton drivers, like the reference's global
 * selected_preconditioner (solvers/options.cpp:8): kind 0 Jacobi, 1 block-Jacobi with
 * block_size rows per block (the reference's kJacobiBlockSize is 8). */
void or_set_preconditioner(int32_t kind, int32_t block_size);

/* Block-Jacobi inverses (block_jacobi_preconditioner.cu:72-167), blocks of bs rows:
 * inv[(b * bs + j) * bs + i] = (block b)^-1 (i, j); unusable block: inv[b*bs*bs] = NaN. */
int or_block_jacobi(int32_t n, const int32_t *row_offsets, const int32_t *columns,
                    const double *values, const double *diagonal, int32_t bs, double *inv,
                    int32_t *fallback_blocks);

/* PCG with the diagonal (blocks == NULL) or block-Jacobi preconditioner. */
int or_pcg_block(int32_t n, const int32_t *row_offsets, const int32_t *columns,
                 const double *values, const double *diagonal, const double *rhs,
                 double tolerance, int32_t max_iterations, const double *blocks, int32_t bs,
                 double *x, int32_t *iterations, double *residual_l2);

/* Deterministic PCG as run by DeterministicPcgKernel (pcg_kernels.cu:10-344) with the
 * preconditioner chosen by or_set_preconditioner. */
int or_pcg(int32_t n, const int32_t *row_offsets, const int32_t *columns, const double *values,
           const double *diagonal, const double *rhs, double tolerance, int32_t max_iterations,
           double *x, int32_t *iterations, double *residual_l2);

/* Newton driver (nonlinear_solver.cu:183-530 device-assembly semantics for a batch,
 * :667-769 for a warm start), finalize (:16-83) and recovery (:534-659).
 * currents [k*c]; warm [k*N] or NULL; outputs a[k*N], b1/b2[k*E], flux[k*c], info[k]. */
int or_solve_batch(const or_model *m, int32_t items, const double *currents, const double *warm,
                   const or_options *options, double *a, double *b1, double *b2, double *flux,
                   or_info *info);

/* B and flux recovery for a given nodal solution (nonlinear_solver.cu:16-83). */
int or_finalize(const or_model *m, const double *a, double *b1, double *b2, double *flux);

#ifdef __cplusplus
}
#endif
#endif
