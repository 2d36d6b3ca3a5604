/*
 * femm_oracle.c -- CPU restatement of FEMM-GPU's nonlinear magnetostatic path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py.  It is never linked into the product.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the FEMM-GPU repository root).  Summation orders follow the reference host
 * code so that oracle/_ref (the reference sources compiled here) reproduces the
 * assembled systems bit for bit; the PCG follows the GPU kernel's algorithm
 * with serial (not tree) reductions.
 */
#include "femm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.141592653589793238462643383279502884
#define OR_TWO_PI 6.283185307179586476925286766559005768
#define OR_MU0 (4.0e-7 * OR_PI)

/* ------------------------------------------------------------------------- */
/* B-H spline: gpu_solver/src/physics/nonlinear_model.cpp:13-113              */
/* ------------------------------------------------------------------------- */

/* Natural-cubic slope system of FEMM's DC GetSlopes, solved by Gaussian
 * elimination with partial pivoting.  The matrix is tridiagonal, so only the
 * band is touched; the arithmetic is the same as the dense elimination since
 * the skipped updates all subtract exact zeros. */
static int bh_slopes(int n, const double *b, const double *h, double *slope)
{
  /* Band storage of rows that may grow one extra super-diagonal under pivoting. */
  double *lo = calloc((size_t)n, sizeof(double)); /* a[i][i-1] */
  double *di = calloc((size_t)n, sizeof(double)); /* a[i][i]   */
  double *up = calloc((size_t)n, sizeof(double)); /* a[i][i+1] */
  double *u2 = calloc((size_t)n, sizeof(double)); /* a[i][i+2] (fill from swaps) */
  double *rhs = calloc((size_t)n, sizeof(double));
  int ok = 1;
  if (!lo || !di || !up || !u2 || !rhs) {
    ok = 0;
    goto done;
  }
  {
    const double first = b[1] - b[0];
    di[0] = 4.0 / first;
    up[0] = 2.0 / first;
    rhs[0] = 6.0 * (h[1] - h[0]) / (first * first);
    const double last = b[n - 1] - b[n - 2];
    di[n - 1] = 4.0 / last;
    lo[n - 1] = 2.0 / last;
    rhs[n - 1] = 6.0 * (h[n - 1] - h[n - 2]) / (last * last);
    for (int i = 1; i < n - 1; ++i) {
      const double left = b[i] - b[i - 1];
      const double right = b[i + 1] - b[i];
      lo[i] = 2.0 / left;
      di[i] = 4.0 * (left + right) / (left * right);
      up[i] = 2.0 / right;
      rhs[i] = 6.0 * (h[i] - h[i - 1]) / (left * left) + 6.0 * (h[i + 1] - h[i]) / (right * right);
    }
  }
  for (int pc = 0; pc < n; ++pc) {
    /* Candidates for the pivot: row pc (diagonal) and row pc+1 (sub-diagonal). */
    if (pc + 1 < n && fabs(lo[pc + 1]) > fabs(di[pc])) {
      /* Swap rows pc and pc+1 in columns >= pc. Row pc holds (di, up, u2), row pc+1
       * holds (lo, di, up) at columns (pc, pc+1, pc+2). */
      double r0 = di[pc], r1 = up[pc], r2 = u2[pc];
      double s0 = lo[pc + 1], s1 = di[pc + 1], s2 = up[pc + 1];
      di[pc] = s0; up[pc] = s1; u2[pc] = s2;
      lo[pc + 1] = r0; di[pc + 1] = r1; up[pc + 1] = r2;
      double t = rhs[pc]; rhs[pc] = rhs[pc + 1]; rhs[pc + 1] = t;
    }
    if (!(fabs(di[pc]) > 0.0)) {
      ok = 0;
      goto done;
    }
    if (pc + 1 < n) {
      const double factor = lo[pc + 1] / di[pc];
      lo[pc + 1] -= factor * di[pc];
      di[pc + 1] -= factor * up[pc];
      up[pc + 1] -= factor * u2[pc];
      rhs[pc + 1] -= factor * rhs[pc];
    }
  }
  for (int row = n - 1; row >= 0; --row) {
    double value = rhs[row];
    if (row + 1 < n)
      value -= up[row] * slope[row + 1];
    if (row + 2 < n)
      value -= u2[row] * slope[row + 2];
    slope[row] = value / di[row];
    if (!isfinite(slope[row])) {
      ok = 0;
      goto done;
    }
  }
done:
  free(lo); free(di); free(up); free(u2); free(rhs);
  return ok;
}

int or_bh_build(int32_t n, double *b, double *h, double *slope, double *cold_secant,
                int32_t *smoothing_passes)
{
  if (n < 2 || b[0] != 0.0 || h[0] != 0.0)
    return 0;
  if (!(*cold_secant > 0.0))
    *cold_secant = h[1] / b[1];
  for (;;) {
    for (int i = 1; i < n; ++i)
      if (!(b[i] > b[i - 1]) || h[i] < 0.0 || !isfinite(b[i]) || !isfinite(h[i]))
        return 0;
    for (int i = 0; i < n; ++i)
      slope[i] = 0.0;
    if (!bh_slopes(n, b, h, slope))
      return 0;
    int monotone = 1;
    for (int i = 1; i < n; ++i) {
      const double length = b[i] - b[i - 1];
      const double d0 = slope[i - 1], d1 = slope[i];
      const double h0 = h[i - 1], h1 = h[i];
      const double c0 = d0;
      const double c1 = -2.0 * (2.0 * d0 * length + d1 * length + 3.0 * h0 - 3.0 * h1) / (length * length);
      const double c2 = 3.0 * (d0 * length + d1 * length + 2.0 * h0 - 2.0 * h1) / (length * length * length);
      double root0 = -1.0, root1 = -1.0;
      const double disc = c1 * c1 - 4.0 * c0 * c2;
      if (c2 == 0.0) {
        if (c1 != 0.0)
          root0 = -c0 / c1;
      } else if (disc > 0.0) {
        const double root = sqrt(disc);
        root0 = -(c1 + root) / (2.0 * c2);
        root1 = (-c1 + root) / (2.0 * c2);
      }
      if ((root0 >= 0.0 && root0 <= length) || (root1 >= 0.0 && root1 <= length)) {
        monotone = 0;
        break;
      }
    }
    if (monotone)
      return 1;
    if (++*smoothing_passes > 1024)
      return 0;
    double *nb = malloc((size_t)n * sizeof(double)), *nh = malloc((size_t)n * sizeof(double));
    memcpy(nb, b, (size_t)n * sizeof(double));
    memcpy(nh, h, (size_t)n * sizeof(double));
    for (int i = 1; i < n - 1; ++i) {
      nb[i] = (b[i - 1] + b[i] + b[i + 1]) / 3.0;
      nh[i] = (h[i - 1] + h[i] + h[i + 1]) / 3.0;
    }
    memcpy(b, nb, (size_t)n * sizeof(double));
    memcpy(h, nh, (size_t)n * sizeof(double));
    free(nb);
    free(nh);
  }
}

/* nonlinear_model.cpp:115-148 */
void or_bh_eval(int32_t n, const double *bt, const double *ht, const double *slope, double field_b,
                double *out)
{
  double hv = 0.0, dh = 0.0, nu = 0.0, dnu = 0.0;
  const double b = fabs(field_b);
  if (b == 0.0) {
    out[0] = 0.0;
    out[1] = slope[0];
    out[2] = slope[0];
    out[3] = 0.0;
    return;
  }
  if (b > bt[n - 1]) {
    hv = ht[n - 1] + slope[n - 1] * (b - bt[n - 1]);
    dh = slope[n - 1];
  } else {
    for (int i = 0; i < n - 1; ++i) {
      if (b >= bt[i] && b <= bt[i + 1]) {
        const double length = bt[i + 1] - bt[i];
        const double z = (b - bt[i]) / length, z2 = z * z;
        hv = (1.0 - 3.0 * z2 + 2.0 * z2 * z) * ht[i] + z * (1.0 - 2.0 * z + z2) * length * slope[i] +
             z2 * (3.0 - 2.0 * z) * ht[i + 1] + z2 * (z - 1.0) * length * slope[i + 1];
        dh = 6.0 * z * (z - 1.0) * ht[i] / length + (1.0 - 4.0 * z + 3.0 * z2) * slope[i] +
             6.0 * z * (1.0 - z) * ht[i + 1] / length + z * (3.0 * z - 2.0) * slope[i + 1];
        break;
      }
    }
  }
  nu = hv / b;
  dnu = 0.5 * (dh / (b * b) - hv / (b * b * b));
  out[0] = hv;
  out[1] = dh;
  out[2] = nu;
  out[3] = dnu;
}

/* ------------------------------------------------------------------------- */
/* Signed DOF map: gpu_solver/src/signed_node_constraints.h:33-106            */
/* ------------------------------------------------------------------------- */
int or_signed_dofs(int32_t N, int32_t nc, const int32_t *ca, const int32_t *cb, const int8_t *cs,
                   int32_t nd, const int32_t *dn, const double *dv, int32_t *node_root,
                   int8_t *node_sign, int32_t *node_to_free, double *boundary_values,
                   int32_t *free_count)
{
  if (N <= 0)
    return 3;
  /* Adjacency in constraint order: for each constraint, a->b then b->a. */
  int32_t *deg = calloc((size_t)N + 1, sizeof(int32_t));
  for (int i = 0; i < nc; ++i) {
    if (ca[i] < 0 || cb[i] < 0 || ca[i] >= N || cb[i] >= N || (cs[i] != 1 && cs[i] != -1)) {
      free(deg);
      return 1;
    }
    if (ca[i] == cb[i]) {
      free(deg);
      return cs[i] < 0 ? 2 : 1;
    }
    deg[ca[i] + 1]++;
    deg[cb[i] + 1]++;
  }
  for (int i = 0; i < N; ++i)
    deg[i + 1] += deg[i];
  int32_t *adj = malloc(sizeof(int32_t) * (size_t)(deg[N] + 1));
  int8_t *adjs = malloc((size_t)(deg[N] + 1));
  int32_t *fill = calloc((size_t)N, sizeof(int32_t));
  for (int i = 0; i < nc; ++i) {
    int p = deg[ca[i]] + fill[ca[i]]++;
    adj[p] = cb[i];
    adjs[p] = cs[i];
    p = deg[cb[i]] + fill[cb[i]]++;
    adj[p] = ca[i];
    adjs[p] = cs[i];
  }
  int rc = 0;
  int32_t *stack = malloc(sizeof(int32_t) * (size_t)N);
  for (int i = 0; i < N; ++i) {
    node_root[i] = -1;
    node_sign[i] = 0;
  }
  for (int start = 0; start < N && rc == 0; ++start) {
    if (node_root[start] >= 0)
      continue;
    node_root[start] = start;
    node_sign[start] = 1;
    int top = 0;
    stack[top++] = start;
    while (top > 0 && rc == 0) {
      const int node = stack[--top];
      for (int e = deg[node]; e < deg[node + 1]; ++e) {
        const int nb = adj[e];
        const int8_t s = (int8_t)(node_sign[node] * adjs[e]);
        if (node_root[nb] < 0) {
          node_root[nb] = start;
          node_sign[nb] = s;
          stack[top++] = nb;
        } else if (node_root[nb] != start || node_sign[nb] != s) {
          rc = 2;
          break;
        }
      }
    }
  }
  char *fixed = calloc((size_t)N, 1);
  double *root_value = calloc((size_t)N, sizeof(double));
  for (int i = 0; i < nd && rc == 0; ++i) {
    const int node = dn[i];
    const double value = dv[i];
    if (node < 0 || node >= N || !isfinite(value)) {
      rc = 3;
      break;
    }
    const int root = node_root[node];
    const double rv = (double)node_sign[node] * value;
    if (fixed[root] && root_value[root] != rv) {
      rc = 3;
      break;
    }
    fixed[root] = 1;
    root_value[root] = rv;
  }
  if (rc == 0) {
    int32_t nf = 0;
    int32_t *root_to_free = malloc(sizeof(int32_t) * (size_t)N);
    for (int i = 0; i < N; ++i) {
      root_to_free[i] = -1;
      if (node_root[i] == i && !fixed[i])
        root_to_free[i] = nf++;
    }
    for (int i = 0; i < N; ++i) {
      const int root = node_root[i];
      node_to_free[i] = root_to_free[root];
      boundary_values[i] = fixed[root] ? (double)node_sign[i] * root_value[root] : 0.0;
    }
    *free_count = nf;
    free(root_to_free);
  }
  free(deg); free(adj); free(adjs); free(fill); free(stack); free(fixed); free(root_value);
  return rc;
}

/* ------------------------------------------------------------------------- */
/* Element terms                                                              */
/* ------------------------------------------------------------------------- */

/* nonlinear_model.cpp:207-221 */
static int element_terms(const double *p0, const double *p1, const double *p2, double *area,
                         double bx[3], double by[3])
{
  const double det = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
  if (!(det > 0.0) || !isfinite(det))
    return 0;
  *area = 0.5 * det;
  const double dx[3] = {p1[1] - p2[1], p2[1] - p0[1], p0[1] - p1[1]};
  const double dy[3] = {p2[0] - p1[0], p0[0] - p2[0], p1[0] - p0[0]};
  for (int i = 0; i < 3; ++i) {
    bx[i] = dy[i] / det;
    by[i] = -dx[i] / det;
  }
  return 1;
}

/* Seven-point Dunavant rule (axisymmetric_p1.h:47-60): published quadrature table. */
static const double kBary[7][3] = {
    {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0},
    {0.059715871789770, 0.470142064105115, 0.470142064105115},
    {0.470142064105115, 0.059715871789770, 0.470142064105115},
    {0.470142064105115, 0.470142064105115, 0.059715871789770},
    {0.797426985353087, 0.101286507323456, 0.101286507323456},
    {0.101286507323456, 0.797426985353087, 0.101286507323456},
    {0.101286507323456, 0.101286507323456, 0.797426985353087},
};
static const double kQw[7] = {0.225, 0.132394152788506, 0.132394152788506, 0.132394152788506,
                              0.125939180544827, 0.125939180544827, 0.125939180544827};

typedef struct {
  double area;
  double w[7], r[7], shape[7][3], br[7][3], bz[7][3];
} axi_elem;

/* axisymmetric_p1.h:26-77 */
static int axi_element(const double r[3], const double z[3], axi_elem *e)
{
  const double det = (r[1] - r[0]) * (z[2] - z[0]) - (r[2] - r[0]) * (z[1] - z[0]);
  if (!(det > 0.0) || !isfinite(det))
    return 0;
  const double dndr[3] = {(z[1] - z[2]) / det, (z[2] - z[0]) / det, (z[0] - z[1]) / det};
  const double dndz[3] = {(r[2] - r[1]) / det, (r[0] - r[2]) / det, (r[1] - r[0]) / det};
  e->area = 0.5 * det;
  for (int p = 0; p < 7; ++p) {
    e->w[p] = e->area * kQw[p];
    e->r[p] = 0.0;
    for (int l = 0; l < 3; ++l) {
      e->shape[p][l] = kBary[p][l];
      e->r[p] += e->shape[p][l] * r[l];
    }
    if (!(e->r[p] > 0.0) || !isfinite(e->r[p]))
      return 0;
    for (int l = 0; l < 3; ++l) {
      e->br[p][l] = -dndz[l];
      e->bz[p][l] = dndr[l] + e->shape[p][l] / e->r[p];
    }
  }
  return 1;
}

/* ------------------------------------------------------------------------- */
/* Built model: processed curves and the signed map                           */
/* ------------------------------------------------------------------------- */
typedef struct {
  const or_model *m;
  or_curve *curves;
  int32_t *node_root, *node_to_free;
  int8_t *node_sign;
  double *boundary;
  int32_t *free_nodes;
  int32_t free_count;
  int has_nonlinear;
} built_model;

static void built_free(built_model *bm)
{
  if (bm->curves) {
    for (int c = 0; c < bm->m->curve_count; ++c) {
      free(bm->curves[c].b);
      free(bm->curves[c].h);
      free(bm->curves[c].slope);
    }
    free(bm->curves);
  }
  free(bm->node_root); free(bm->node_to_free); free(bm->node_sign); free(bm->boundary);
  free(bm->free_nodes);
  memset(bm, 0, sizeof(*bm));
}

/* nonlinear_model.cpp:223-319 (validation) */
int or_validate(const or_model *m)
{
  if (m->node_count <= 0 || m->tri_count <= 0 || m->mat_count <= 0 ||
      (m->problem_type == 0 && (!(m->depth_m > 0.0) || !isfinite(m->depth_m))) ||
      m->circuit_count < 0 || m->dir_count <= 0)
    return OR_INVALID_ARGUMENT;
  if (m->age_count != 0)
    return OR_UNSUPPORTED; /* air-gap elements: checked against the reference build only */
  char *bnd = calloc((size_t)m->node_count, 1);
  for (int i = 0; i < m->dir_count; ++i) {
    const int node = m->dir_nodes[i];
    if (node < 0 || node >= m->node_count || bnd[node] || !isfinite(m->dir_values[i])) {
      free(bnd);
      return OR_BOUNDARY_INVALID;
    }
    bnd[node] = 1;
  }
  free(bnd);
  if (m->dir_count == m->node_count)
    return OR_BOUNDARY_INVALID;
  for (int i = 0; i < m->node_count; ++i)
    if (!isfinite(m->xy[2 * i]) || !isfinite(m->xy[2 * i + 1]) ||
        (m->problem_type == 1 && m->xy[2 * i] < 0.0))
      return OR_MESH_INVALID;
  for (int i = 0; i < m->mat_count; ++i) {
    if (!(m->nu0[i] > 0.0) || m->alpha[i] < 0.0 || !isfinite(m->nu0[i]) || !isfinite(m->alpha[i]) ||
        !isfinite(m->j_per_a[i]) || !isfinite(m->hc[i]) || !isfinite(m->mag_deg[i]))
      return OR_INVALID_MATERIAL;
    if (m->circuit_index[i] < -1 || m->circuit_index[i] >= m->circuit_count ||
        (m->j_per_a[i] != 0.0 && m->circuit_index[i] < 0))
      return OR_INVALID_MATERIAL;
    if (m->curve_index[i] < -1 || m->curve_index[i] >= m->curve_count)
      return OR_INVALID_MATERIAL;
  }
  for (int e = 0; e < m->tri_count; ++e) {
    if (m->tri_mat[e] < 0 || m->tri_mat[e] >= m->mat_count)
      return OR_INVALID_MATERIAL;
    for (int l = 0; l < 3; ++l)
      if (m->tri[3 * e + l] < 0 || m->tri[3 * e + l] >= m->node_count)
        return OR_MESH_INVALID;
    double area, bx[3], by[3];
    if (!element_terms(m->xy + 2 * m->tri[3 * e], m->xy + 2 * m->tri[3 * e + 1],
                       m->xy + 2 * m->tri[3 * e + 2], &area, bx, by))
      return OR_MESH_INVALID;
  }
  return OR_OK;
}

static int build_model(const or_model *m, built_model *bm)
{
  memset(bm, 0, sizeof(*bm));
  bm->m = m;
  int status = or_validate(m);
  if (status != OR_OK)
    return status;
  bm->curves = calloc((size_t)(m->curve_count > 0 ? m->curve_count : 1), sizeof(or_curve));
  for (int c = 0; c < m->curve_count; ++c) {
    const int off = m->curve_offsets[c], cnt = m->curve_offsets[c + 1] - m->curve_offsets[c];
    or_curve *cv = &bm->curves[c];
    cv->count = cnt;
    cv->b = malloc(sizeof(double) * (size_t)(cnt > 0 ? cnt : 1));
    cv->h = malloc(sizeof(double) * (size_t)(cnt > 0 ? cnt : 1));
    cv->slope = calloc((size_t)(cnt > 0 ? cnt : 1), sizeof(double));
    memcpy(cv->b, m->curve_b + off, sizeof(double) * (size_t)cnt);
    memcpy(cv->h, m->curve_h + off, sizeof(double) * (size_t)cnt);
    cv->cold_secant = 0.0;
    if (!or_bh_build(cnt, cv->b, cv->h, cv->slope, &cv->cold_secant, &cv->smoothing_passes)) {
      built_free(bm);
      return OR_INVALID_MATERIAL;
    }
  }
  const int N = m->node_count;
  bm->node_root = malloc(sizeof(int32_t) * (size_t)N);
  bm->node_to_free = malloc(sizeof(int32_t) * (size_t)N);
  bm->node_sign = malloc((size_t)N);
  bm->boundary = malloc(sizeof(double) * (size_t)N);
  if (or_signed_dofs(N, m->con_count, m->con_a, m->con_b, m->con_sign, m->dir_count, m->dir_nodes,
                     m->dir_values, bm->node_root, bm->node_sign, bm->node_to_free, bm->boundary,
                     &bm->free_count) != 0 ||
      bm->free_count == 0) {
    built_free(bm);
    return OR_BOUNDARY_INVALID;
  }
  bm->free_nodes = malloc(sizeof(int32_t) * (size_t)bm->free_count);
  for (int i = 0; i < N; ++i)
    if (bm->node_root[i] == i && bm->node_to_free[i] >= 0)
      bm->free_nodes[bm->node_to_free[i]] = i;
  if (m->problem_type == 1) {
    double scale = 1e-3;
    for (int i = 0; i < N; ++i)
      if (m->xy[2 * i] > scale)
        scale = m->xy[2 * i];
    const double tol = 1e-12 * scale;
    for (int i = 0; i < N; ++i)
      if (m->xy[2 * i] <= tol && (bm->node_to_free[i] >= 0 || bm->boundary[i] != 0.0)) {
        built_free(bm);
        return OR_BOUNDARY_INVALID;
      }
  }
  bm->has_nonlinear = 0;
  for (int i = 0; i < m->mat_count; ++i)
    if (m->curve_index[i] >= 0 || m->alpha[i] != 0.0)
      bm->has_nonlinear = 1;
  return OR_OK;
}

/* nonlinear_model.cpp:428-451 */
static int material_eval(const built_model *bm, int mat, double bmag, int use_newton, double *nu,
                         double *dnu)
{
  const or_model *m = bm->m;
  const int c = m->curve_index[mat];
  double ev[4] = {0, 0, 0, 0};
  if (c >= 0) {
    const or_curve *cv = &bm->curves[c];
    or_bh_eval(cv->count, cv->b, cv->h, cv->slope, bmag, ev);
    *nu = ev[2];
  } else {
    *nu = m->nu0[mat] * (1.0 + m->alpha[mat] * bmag * bmag);
  }
  *dnu = use_newton ? (c >= 0 ? ev[3] : m->nu0[mat] * m->alpha[mat]) : 0.0;
  if (!use_newton && c >= 0)
    *nu = bm->curves[c].cold_secant;
  return *nu > 0.0 && isfinite(*nu) && isfinite(*dnu);
}

/* ------------------------------------------------------------------------- */
/* Sparse row storage with sorted columns (std::map semantics)               */
/* ------------------------------------------------------------------------- */
typedef struct {
  int32_t rows;
  int32_t *off; /* rows + 1 */
  int32_t *col;
  double *val;
} csr;

static int cmp_i32(const void *a, const void *b)
{
  const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* Build a row-sorted unique pattern from per-row candidate lists. */
static void csr_finish(csr *s, int32_t *cand_off, int32_t *cand)
{
  s->off = malloc(sizeof(int32_t) * (size_t)(s->rows + 1));
  int32_t total = 0;
  for (int r = 0; r < s->rows; ++r) {
    int32_t *row = cand + cand_off[r];
    const int len = cand_off[r + 1] - cand_off[r];
    qsort(row, (size_t)len, sizeof(int32_t), cmp_i32);
    int u = 0;
    for (int k = 0; k < len; ++k)
      if (u == 0 || row[u - 1] != row[k])
        row[u++] = row[k];
    s->off[r] = total;
    total += u;
    cand_off[r] = u; /* reuse as unique length */
  }
  s->off[s->rows] = total;
  s->col = malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  s->val = calloc((size_t)(total > 0 ? total : 1), sizeof(double));
  /* cand_off now holds lengths; recover starts from the running candidate layout */
  return;
}

static int32_t csr_find(const csr *s, int32_t r, int32_t c)
{
  int lo = s->off[r], hi = s->off[r + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (s->col[mid] == c)
      return mid;
    if (s->col[mid] < c)
      lo = mid + 1;
    else
      hi = mid - 1;
  }
  return -1;
}

static void csr_free(csr *s)
{
  free(s->off);
  free(s->col);
  free(s->val);
  memset(s, 0, sizeof(*s));
}

/* Pattern builder: pairs (r, c) listed per row, then sorted/uniqued. */
static void csr_from_pairs(csr *s, int32_t rows, int64_t npairs, const int32_t *pr,
                           const int32_t *pc)
{
  s->rows = rows;
  int32_t *cnt = calloc((size_t)rows + 1, sizeof(int32_t));
  for (int64_t k = 0; k < npairs; ++k)
    cnt[pr[k] + 1]++;
  for (int r = 0; r < rows; ++r)
    cnt[r + 1] += cnt[r];
  int32_t *start = malloc(sizeof(int32_t) * ((size_t)rows + 1));
  memcpy(start, cnt, sizeof(int32_t) * ((size_t)rows + 1));
  int32_t *cand = malloc(sizeof(int32_t) * (size_t)(npairs > 0 ? npairs : 1));
  int32_t *fill = calloc((size_t)rows, sizeof(int32_t));
  for (int64_t k = 0; k < npairs; ++k)
    cand[cnt[pr[k]] + fill[pr[k]]++] = pc[k];
  csr_finish(s, cnt, cand);
  for (int r = 0; r < rows; ++r)
    memcpy(s->col + s->off[r], cand + start[r], sizeof(int32_t) * (size_t)cnt[r]);
  free(cnt);
  free(start);
  free(cand);
  free(fill);
}

/* ------------------------------------------------------------------------- */
/* Host Newton assembler: nonlinear_model.cpp:453-627, reduction :321-394     */
/* ------------------------------------------------------------------------- */
struct or_system {
  int32_t rows, nnz, circuits, N;
  int32_t *off, *col;
  double *val, *diag, *rhs_per_amp, *rhs_offset;
  double *circuit_src; /* [c * rows]: signed-reduced per-circuit source loads */
  int32_t *node_to_free, *free_nodes;
  int8_t *node_sign;
  double *boundary;
};

void or_system_free(or_system *s)
{
  if (!s)
    return;
  free(s->off); free(s->col); free(s->val); free(s->diag); free(s->rhs_per_amp);
  free(s->rhs_offset); free(s->circuit_src); free(s->node_to_free); free(s->free_nodes);
  free(s->node_sign); free(s->boundary);
  free(s);
}

int32_t or_system_rows(const or_system *s) { return s->rows; }
int32_t or_system_nnz(const or_system *s) { return s->nnz; }

void or_system_copy(const or_system *s, int32_t *row_offsets, int32_t *columns, double *values,
                    double *diagonal, double *rhs, int32_t *node_to_free, int8_t *node_sign,
                    double *boundary_values, double *circuit_sources)
{
  if (row_offsets)
    memcpy(row_offsets, s->off, sizeof(int32_t) * (size_t)(s->rows + 1));
  if (columns)
    memcpy(columns, s->col, sizeof(int32_t) * (size_t)s->nnz);
  if (values)
    memcpy(values, s->val, sizeof(double) * (size_t)s->nnz);
  if (diagonal)
    memcpy(diagonal, s->diag, sizeof(double) * (size_t)s->rows);
  if (rhs)
    for (int r = 0; r < s->rows; ++r)
      rhs[r] = s->rhs_per_amp[r] + s->rhs_offset[r];
  if (node_to_free)
    memcpy(node_to_free, s->node_to_free, sizeof(int32_t) * (size_t)s->N);
  if (node_sign)
    memcpy(node_sign, s->node_sign, (size_t)s->N);
  if (boundary_values)
    memcpy(boundary_values, s->boundary, sizeof(double) * (size_t)s->N);
  if (circuit_sources)
    memcpy(circuit_sources, s->circuit_src, sizeof(double) * (size_t)s->circuits * (size_t)s->rows);
}

static int assemble_built(const built_model *bm, const double *a_old, const double *currents,
                          int use_newton, or_system **out)
{
  const or_model *m = bm->m;
  const int N = m->node_count, E = m->tri_count, C = m->circuit_count;
  *out = NULL;
  for (int c = 0; c < C; ++c)
    if (!isfinite(currents[c]))
      return OR_INVALID_ARGUMENT;
  /* Full (node x node) pattern from every triangle couple. */
  int32_t *pr = malloc(sizeof(int32_t) * (size_t)E * 9), *pc = malloc(sizeof(int32_t) * (size_t)E * 9);
  for (int e = 0; e < E; ++e)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        pr[9 * e + 3 * i + j] = m->tri[3 * e + i];
        pc[9 * e + 3 * i + j] = m->tri[3 * e + j];
      }
  csr full;
  csr_from_pairs(&full, N, (int64_t)E * 9, pr, pc);
  free(pr);
  free(pc);
  double *rhs = calloc((size_t)N, sizeof(double));
  double *src = calloc((size_t)N * (size_t)(C > 0 ? C : 1), sizeof(double));
  int status = OR_OK;
  for (int e = 0; e < E && status == OR_OK; ++e) {
    const int mat = m->tri_mat[e];
    const int *tn = m->tri + 3 * e;
    const double theta = m->mag_deg[mat] * OR_PI / 180.0;
    const double hcx = m->hc[mat] * cos(theta), hcy = m->hc[mat] * sin(theta);
    const int circuit = m->circuit_index[mat];
    const double jpa = m->j_per_a[mat];
    if (m->problem_type == 0) {
      double area, bxv[3], byv[3];
      if (!element_terms(m->xy + 2 * tn[0], m->xy + 2 * tn[1], m->xy + 2 * tn[2], &area, bxv, byv)) {
        status = OR_MESH_INVALID;
        break;
      }
      double bx = 0.0, by = 0.0;
      for (int i = 0; i < 3; ++i) {
        bx += a_old[tn[i]] * bxv[i];
        by += a_old[tn[i]] * byv[i];
      }
      double nu, dnu;
      if (!material_eval(bm, mat, hypot(bx, by), use_newton, &nu, &dnu)) {
        status = OR_NONFINITE;
        break;
      }
      for (int i = 0; i < 3 && status == OR_OK; ++i) {
        const int gi = tn[i];
        const double coil = area * jpa / 3.0;
        const double pm = area * (hcx * bxv[i] + hcy * byv[i]);
        if (circuit >= 0) {
          src[(size_t)circuit * N + gi] += coil;
          rhs[gi] += currents[circuit] * coil;
        }
        rhs[gi] += pm;
        const double bdi = bx * bxv[i] + by * byv[i];
        for (int j = 0; j < 3; ++j) {
          const int gj = tn[j];
          const double bdj = bx * bxv[j] + by * byv[j];
          const double k = area * nu * (bxv[i] * bxv[j] + byv[i] * byv[j]);
          const double c = use_newton ? 2.0 * area * dnu * bdi * bdj : 0.0;
          const double v = k + c;
          const int32_t slot = csr_find(&full, gi, gj);
          if (!isfinite(v)) {
            status = OR_NONFINITE;
            break;
          }
          full.val[slot] += v;
          if (!isfinite(full.val[slot])) {
            status = OR_NONFINITE;
            break;
          }
          if (use_newton)
            rhs[gi] += c * a_old[gj];
        }
      }
    } else {
      const double r[3] = {m->xy[2 * tn[0]], m->xy[2 * tn[1]], m->xy[2 * tn[2]]};
      const double z[3] = {m->xy[2 * tn[0] + 1], m->xy[2 * tn[1] + 1], m->xy[2 * tn[2] + 1]};
      axi_elem ax;
      if (!axi_element(r, z, &ax)) {
        status = OR_MESH_INVALID;
        break;
      }
      for (int p = 0; p < 7 && status == OR_OK; ++p) {
        double br = 0.0, bz = 0.0;
        for (int l = 0; l < 3; ++l) {
          const double v = a_old[tn[l]];
          br += v * ax.br[p][l];
          bz += v * ax.bz[p][l];
        }
        double nu, dnu;
        if (!material_eval(bm, mat, hypot(br, bz), use_newton, &nu, &dnu)) {
          status = OR_NONFINITE;
          break;
        }
        const double vw = OR_TWO_PI * ax.r[p] * ax.w[p];
        for (int i = 0; i < 3 && status == OR_OK; ++i) {
          const int gi = tn[i];
          const double coil = vw * jpa * ax.shape[p][i];
          const double pm = vw * (hcx * ax.br[p][i] + hcy * ax.bz[p][i]);
          if (circuit >= 0) {
            src[(size_t)circuit * N + gi] += coil;
            rhs[gi] += currents[circuit] * coil;
          }
          rhs[gi] += pm;
          const double bdi = br * ax.br[p][i] + bz * ax.bz[p][i];
          for (int j = 0; j < 3; ++j) {
            const int gj = tn[j];
            const double bdj = br * ax.br[p][j] + bz * ax.bz[p][j];
            const double k = vw * nu * (ax.br[p][i] * ax.br[p][j] + ax.bz[p][i] * ax.bz[p][j]);
            const double c = use_newton ? 2.0 * vw * dnu * bdi * bdj : 0.0;
            const double v = k + c;
            const int32_t slot = csr_find(&full, gi, gj);
            if (!isfinite(v)) {
              status = OR_NONFINITE;
              break;
            }
            full.val[slot] += v;
            if (!isfinite(full.val[slot])) {
              status = OR_NONFINITE;
              break;
            }
            if (use_newton)
              rhs[gi] += c * a_old[gj];
          }
        }
      }
    }
  }
  if (status != OR_OK) {
    csr_free(&full);
    free(rhs);
    free(src);
    return status;
  }
  /* Signed reduction T^T K T (nonlinear_model.cpp:321-394). */
  const int R = bm->free_count;
  or_system *s = calloc(1, sizeof(or_system));
  s->rows = R;
  s->circuits = C;
  s->N = N;
  int64_t np = 0;
  for (int node = 0; node < N; ++node) {
    if (bm->node_to_free[node] < 0)
      continue;
    for (int k = full.off[node]; k < full.off[node + 1]; ++k)
      if (bm->node_to_free[full.col[k]] >= 0)
        ++np;
  }
  int32_t *rr = malloc(sizeof(int32_t) * (size_t)(np > 0 ? np : 1));
  int32_t *rc = malloc(sizeof(int32_t) * (size_t)(np > 0 ? np : 1));
  np = 0;
  for (int node = 0; node < N; ++node) {
    const int row = bm->node_to_free[node];
    if (row < 0)
      continue;
    for (int k = full.off[node]; k < full.off[node + 1]; ++k) {
      const int col = bm->node_to_free[full.col[k]];
      if (col >= 0) {
        rr[np] = row;
        rc[np] = col;
        ++np;
      }
    }
  }
  csr red;
  csr_from_pairs(&red, R, np, rr, rc);
  free(rr);
  free(rc);
  double *rpa = calloc((size_t)R, sizeof(double)), *roff = calloc((size_t)R, sizeof(double));
  s->circuit_src = calloc((size_t)R * (size_t)(C > 0 ? C : 1), sizeof(double));
  for (int node = 0; node < N && status == OR_OK; ++node) {
    const int row = bm->node_to_free[node];
    if (row < 0)
      continue;
    const double rs = (double)bm->node_sign[node];
    rpa[row] += rs * rhs[node];
    for (int c = 0; c < C; ++c)
      s->circuit_src[(size_t)c * R + row] += rs * src[(size_t)c * N + node];
    for (int k = full.off[node]; k < full.off[node + 1]; ++k) {
      const int cn = full.col[k];
      const int col = bm->node_to_free[cn];
      if (col < 0) {
        roff[row] -= rs * full.val[k] * bm->boundary[cn];
      } else {
        const double v = rs * (double)bm->node_sign[cn] * full.val[k];
        const int32_t slot = csr_find(&red, row, col);
        if (!isfinite(v)) {
          status = OR_NONFINITE;
          break;
        }
        red.val[slot] += v;
        if (!isfinite(red.val[slot])) {
          status = OR_NONFINITE;
          break;
        }
      }
    }
  }
  s->nnz = red.off[R];
  s->off = red.off;
  s->col = red.col;
  s->val = red.val;
  s->diag = calloc((size_t)R, sizeof(double));
  s->rhs_per_amp = rpa;
  s->rhs_offset = roff;
  s->node_to_free = malloc(sizeof(int32_t) * (size_t)N);
  memcpy(s->node_to_free, bm->node_to_free, sizeof(int32_t) * (size_t)N);
  s->node_sign = malloc((size_t)N);
  memcpy(s->node_sign, bm->node_sign, (size_t)N);
  s->boundary = malloc(sizeof(double) * (size_t)N);
  memcpy(s->boundary, bm->boundary, sizeof(double) * (size_t)N);
  s->free_nodes = malloc(sizeof(int32_t) * (size_t)R);
  memcpy(s->free_nodes, bm->free_nodes, sizeof(int32_t) * (size_t)R);
  csr_free(&full);
  free(rhs);
  free(src);
  if (status == OR_OK) {
    for (int r = 0; r < R; ++r) {
      for (int k = s->off[r]; k < s->off[r + 1]; ++k)
        if (s->col[k] == r)
          s->diag[r] = s->val[k];
      if (!(s->diag[r] > 0.0) || !isfinite(s->diag[r]) || !isfinite(rpa[r]) || !isfinite(roff[r])) {
        status = OR_ASSEMBLY_FAILED;
        break;
      }
    }
  }
  if (status != OR_OK) {
    or_system_free(s);
    return status;
  }
  *out = s;
  return OR_OK;
}

int or_assemble(const or_model *m, const double *a_old, const double *currents, int use_newton,
                or_system **out)
{
  built_model bm;
  *out = NULL;
  int status = build_model(m, &bm);
  if (status != OR_OK)
    return status;
  status = assemble_built(&bm, a_old, currents, use_newton, out);
  built_free(&bm);
  return status;
}

/* ------------------------------------------------------------------------- */
/* PCG: DeterministicPcgKernel (gpu_solver/src/solvers/pcg_kernels.cu:10-344) */
/* ------------------------------------------------------------------------- */
static double row_dot(int r, const int32_t *off, const int32_t *col, const double *val,
                      const double *x)
{
  double s = 0.0;
  for (int k = off[r]; k < off[r + 1]; ++k)
    s += val[k] * x[col[k]];
  return s;
}

/* Block-Jacobi preconditioner (block_jacobi_preconditioner.cu:72-167, BuildBlockInverse):
 * per contiguous block of bs rows, the principal block scaled by D^-1/2 is factored by
 * Cholesky and inverted column by column; an unusable block (non-positive or subnormal
 * reciprocal diagonal, asymmetric or non-finite entries, failed pivot, non-finite
 * inverse) is stored as NaN at its first entry and the PCG falls back to the diagonal
 * for its rows.  Storage per block: inv[j * bs + i] = (A_block^-1)(i, j). */
static int g_precond_kind = 0, g_block_size = 8;

void or_set_preconditioner(int32_t kind, int32_t block_size)
{
  g_precond_kind = kind;
  g_block_size = block_size;
}

int or_block_jacobi(int32_t n, const int32_t *off, const int32_t *col, const double *val,
                    const double *diag, int32_t bs, double *inv, int32_t *fallback_blocks)
{
  if (n <= 0 || bs <= 0 || bs > 64)
    return OR_INVALID_ARGUMENT;
  const int blocks = (n + bs - 1) / bs;
  double *f = malloc(sizeof(double) * (size_t)bs * (size_t)bs);
  double *xs = malloc(sizeof(double) * (size_t)bs * (size_t)bs);
  double *sc = malloc(sizeof(double) * (size_t)bs);
  int fallbacks = 0;
  for (int b = 0; b < blocks; ++b) {
    const int first = b * bs, width = n - first < bs ? n - first : bs;
    double *out = inv + (size_t)b * (size_t)bs * (size_t)bs;
    int bad = 0;
    for (int l = 0; l < bs; ++l)
      sc[l] = l < width ? sqrt(diag[first + l]) : 1.0;
    for (int k = 0; k < bs * bs; ++k)
      f[k] = 0.0;
    for (int l = 0; l < width; ++l)
      for (int k = off[first + l]; k < off[first + l + 1]; ++k) {
        const int c = col[k] - first;
        if (c >= 0 && c < width)
          f[l * bs + c] += val[k] / sc[l] / sc[c];
      }
    for (int row = 0; row < width; ++row) {
      const double reciprocal = 1.0 / diag[first + row];
      if (!isfinite(reciprocal) || reciprocal < 2.2250738585072014e-308)
        bad = 1;
      for (int c = 0; c <= row; ++c) {
        const double x = f[row * bs + c], y = f[c * bs + row];
        if (!isfinite(x) || !isfinite(y) ||
            fabs(x - y) > 1e-12 * fmax(1.0, fmax(fabs(x), fabs(y))))
          bad = 1;
      }
    }
    for (int c = 0; c < width && !bad; ++c) {
      double pivot = f[c * bs + c];
      for (int k = 0; k < c; ++k)
        pivot -= f[c * bs + k] * f[c * bs + k];
      if (!(pivot > 0.0) || !isfinite(pivot)) {
        bad = 1;
        break;
      }
      f[c * bs + c] = sqrt(pivot);
      for (int row = c + 1; row < width; ++row) {
        double v = f[row * bs + c];
        for (int k = 0; k < c; ++k)
          v -= f[row * bs + k] * f[c * bs + k];
        f[row * bs + c] = v / f[c * bs + c];
      }
    }
    for (int l = 0; l < width && !bad; ++l) { /* column l of the inverse */
      double *x = xs + (size_t)l * bs;
      for (int row = 0; row < width; ++row) {
        double v = row == l ? 1.0 : 0.0;
        for (int k = 0; k < row; ++k)
          v -= f[row * bs + k] * x[k];
        x[row] = v / f[row * bs + row];
      }
      for (int row = width - 1; row >= 0; --row) {
        double v = x[row];
        for (int k = row + 1; k < width; ++k)
          v -= f[k * bs + row] * x[k];
        x[row] = v / f[row * bs + row];
      }
      for (int row = 0; row < width; ++row) {
        x[row] = x[row] / sc[row] / sc[l];
        if (!isfinite(x[row]))
          bad = 1;
      }
    }
    fallbacks += bad;
    for (int l = 0; l < bs; ++l)
      for (int row = 0; row < bs; ++row)
        out[l * bs + row] = bad ? (row == 0 && l == 0 ? NAN : 0.0)
                                : (row < width && l < width ? xs[(size_t)l * bs + row] : 0.0);
  }
  free(f);
  free(xs);
  free(sc);
  if (fallback_blocks)
    *fallback_blocks = fallbacks;
  return OR_OK;
}

/* z_i = (M^-1 r)_i: the block inverse row (pcg_device.cuh:62-79) or the diagonal. */
static double precond_row(int i, int n, const double *r, const double *diag, const double *inv,
                          int use_inv, const double *blocks, int bs)
{
  if (blocks) {
    const int first = i / bs * bs, width = n - first < bs ? n - first : bs;
    const double *blk = blocks + (size_t)(i / bs) * (size_t)bs * (size_t)bs;
    if (!isnan(blk[0])) {
      double v = 0.0;
      for (int j = 0; j < width; ++j)
        v += blk[j * bs + i % bs] * r[first + j];
      return v;
    }
  }
  return use_inv ? r[i] * inv[i] : r[i] / diag[i];
}

int or_pcg_block(int32_t n, const int32_t *off, const int32_t *col, const double *val,
                 const double *diag, const double *rhs, double tol, int32_t maxit,
                 const double *blocks, int32_t bs, double *x, int32_t *iterations,
                 double *residual_l2);

int or_pcg(int32_t n, const int32_t *off, const int32_t *col, const double *val,
           const double *diag, const double *rhs, double tol, int32_t maxit, double *x,
           int32_t *iterations, double *residual_l2)
{
  if (g_precond_kind == 1 && n > 0) {
    const int bs = g_block_size;
    double *blocks = malloc(sizeof(double) * (size_t)((n + bs - 1) / bs) * bs * bs);
    int fb = 0;
    int st = or_block_jacobi(n, off, col, val, diag, bs, blocks, &fb);
    if (st == OR_OK)
      st = or_pcg_block(n, off, col, val, diag, rhs, tol, maxit, blocks, bs, x, iterations,
                        residual_l2);
    free(blocks);
    return st;
  }
  return or_pcg_block(n, off, col, val, diag, rhs, tol, maxit, NULL, 0, x, iterations,
                      residual_l2);
}

/* Deterministic PCG (pcg_kernels.cu:10-344) with the diagonal or a block-Jacobi
 * preconditioner (blocks = or_block_jacobi output, or NULL). */
int or_pcg_block(int32_t n, const int32_t *off, const int32_t *col, const double *val,
                 const double *diag, const double *rhs, double tol, int32_t maxit,
                 const double *blocks, int32_t bs, double *x, int32_t *iterations,
                 double *residual_l2)
{
  *iterations = 0;
  *residual_l2 = INFINITY;
  if (n <= 0 || maxit < 0 || !(tol > 0.0) || !(tol < 1.0) || !isfinite(tol))
    return OR_INVALID_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (!isfinite(rhs[i]) || !isfinite(diag[i]) || !(diag[i] > 0.0))
      return (!isfinite(rhs[i]) || !isfinite(diag[i])) ? OR_NONFINITE : OR_LINEAR_BREAKDOWN;
  /* Inverse diagonal is used when every reciprocal is normal (options.cpp:176-199). */
  double *inv = malloc(sizeof(double) * (size_t)n);
  int use_inv = 1;
  for (int i = 0; i < n; ++i) {
    inv[i] = 1.0 / diag[i];
    if (!isnormal(inv[i]))
      use_inv = 0;
  }
  double *r = malloc(sizeof(double) * (size_t)n), *z = malloc(sizeof(double) * (size_t)n);
  double *p = malloc(sizeof(double) * (size_t)n), *q = malloc(sizeof(double) * (size_t)n);
  int status = OR_INTERNAL;
#define PREC(i) precond_row(i, n, r, diag, inv, use_inv, blocks, bs)
  for (int i = 0; i < n; ++i)
    x[i] = 0.0;
  double scale = 0.0;
  for (int i = 0; i < n; ++i)
    scale = fmax(scale, fabs(rhs[i]));
  if (scale == 0.0) {
    *residual_l2 = 0.0;
    status = OR_OK;
    goto done;
  }
  double rr0 = 0.0, rho = 0.0;
  for (int i = 0; i < n; ++i)
    r[i] = rhs[i] / scale;
  for (int i = 0; i < n; ++i) {
    z[i] = PREC(i);
    p[i] = z[i];
  }
  for (int i = 0; i < n; ++i) {
    rr0 += r[i] * r[i];
    rho += r[i] * z[i];
  }
  if (!isfinite(rr0) || !isfinite(rho)) {
    status = OR_NONFINITE;
    goto done;
  }
  *residual_l2 = sqrt(rr0);
  const double threshold = tol * sqrt(rr0);
  for (int it = 0; it < maxit; ++it) {
    double pq = 0.0;
    for (int i = 0; i < n; ++i) {
      q[i] = row_dot(i, off, col, val, p);
      pq += p[i] * q[i];
    }
    if (!isfinite(pq) || !isfinite(rho)) {
      status = OR_NONFINITE;
      goto done;
    }
    if (!(pq > 0.0) || !(rho > 0.0)) {
      status = OR_LINEAR_BREAKDOWN;
      goto done;
    }
    const double alpha = rho / pq;
    double rr = 0.0, rz = 0.0;
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      rr += r[i] * r[i];
    }
    for (int i = 0; i < n; ++i) {
      z[i] = PREC(i);
      rz += r[i] * z[i];
    }
    *iterations = it + 1;
    if (!isfinite(rr)) {
      status = OR_NONFINITE;
      goto done;
    }
    *residual_l2 = sqrt(rr);
    if (*residual_l2 <= threshold) {
      double tr = 0.0;
      for (int i = 0; i < n; ++i) {
        r[i] = rhs[i] / scale - row_dot(i, off, col, val, x);
        tr += r[i] * r[i];
      }
      if (!isfinite(tr)) {
        status = OR_NONFINITE;
        goto done;
      }
      *residual_l2 = sqrt(tr);
      if (*residual_l2 <= threshold) {
        for (int i = 0; i < n; ++i) {
          x[i] *= scale;
          if (!isfinite(x[i])) {
            status = OR_NONFINITE;
            goto done;
          }
        }
        *residual_l2 *= scale;
        status = isfinite(*residual_l2) ? OR_OK : OR_NONFINITE;
        goto done;
      }
      /* Restart from the true residual. */
      double rs = 0.0;
      for (int i = 0; i < n; ++i) {
        z[i] = PREC(i);
        p[i] = z[i];
        rs += r[i] * z[i];
      }
      if (!isfinite(rs) || !(rs > 0.0)) {
        status = OR_LINEAR_BREAKDOWN;
        goto done;
      }
      rho = rs;
      continue;
    }
    if (!isfinite(rz) || !(rz > 0.0)) {
      status = OR_LINEAR_BREAKDOWN;
      goto done;
    }
    const double beta = rz / rho;
    for (int i = 0; i < n; ++i)
      p[i] = z[i] + beta * p[i];
    rho = rz;
  }
  {
    double tr = 0.0;
    for (int i = 0; i < n; ++i) {
      r[i] = rhs[i] / scale - row_dot(i, off, col, val, x);
      tr += r[i] * r[i];
    }
    if (!isfinite(tr)) {
      status = OR_NONFINITE;
      goto done;
    }
    for (int i = 0; i < n; ++i) {
      x[i] *= scale;
      if (!isfinite(x[i])) {
        status = OR_NONFINITE;
        goto done;
      }
    }
    *residual_l2 = sqrt(tr) * scale;
    status = isfinite(*residual_l2) ? OR_LINEAR_NOT_CONVERGED : OR_NONFINITE;
  }
done:
#undef PREC
  free(inv); free(r); free(z); free(p); free(q);
  return status;
}

/* ------------------------------------------------------------------------- */
/* Finalize: nonlinear_solver.cu:16-83                                       */
/* ------------------------------------------------------------------------- */
static int finalize_built(const built_model *bm, const double *a, double *b1, double *b2,
                          double *flux)
{
  const or_model *m = bm->m;
  const int C = m->circuit_count;
  for (int c = 0; c < C; ++c)
    flux[c] = 0.0;
  int status = OR_OK;
  for (int e = 0; e < m->tri_count; ++e) {
    const int *tn = m->tri + 3 * e;
    const int mat = m->tri_mat[e];
    const int circuit = m->circuit_index[mat];
    double area, bxv[3], byv[3];
    if (!element_terms(m->xy + 2 * tn[0], m->xy + 2 * tn[1], m->xy + 2 * tn[2], &area, bxv, byv))
      return OR_MESH_INVALID;
    b1[e] = 0.0;
    b2[e] = 0.0;
    if (m->problem_type == 0) {
      for (int i = 0; i < 3; ++i) {
        b1[e] += a[tn[i]] * bxv[i];
        b2[e] += a[tn[i]] * byv[i];
      }
      if (circuit >= 0)
        flux[circuit] += area * m->j_per_a[mat] / 3.0 * (a[tn[0]] + a[tn[1]] + a[tn[2]]);
    } else {
      const double r[3] = {m->xy[2 * tn[0]], m->xy[2 * tn[1]], m->xy[2 * tn[2]]};
      const double z[3] = {m->xy[2 * tn[0] + 1], m->xy[2 * tn[1] + 1], m->xy[2 * tn[2] + 1]};
      axi_elem ax;
      if (!axi_element(r, z, &ax))
        return OR_MESH_INVALID;
      for (int l = 0; l < 3; ++l) {
        b1[e] += a[tn[l]] * ax.br[0][l];
        b2[e] += a[tn[l]] * ax.bz[0][l];
      }
      if (!isfinite(b1[e]) || !isfinite(b2[e]))
        return OR_MESH_INVALID;
      if (circuit >= 0) {
        double f = 0.0;
        for (int p = 0; p < 7; ++p) {
          double av = 0.0;
          for (int l = 0; l < 3; ++l)
            av += ax.shape[p][l] * a[tn[l]];
          f += OR_TWO_PI * ax.r[p] * ax.w[p] * m->j_per_a[mat] * av;
        }
        flux[circuit] += f;
      }
    }
  }
  for (int c = 0; c < C; ++c) {
    if (m->problem_type == 0)
      flux[c] *= m->depth_m;
    if (!isfinite(flux[c]))
      status = OR_NONFINITE;
  }
  return status;
}

int or_finalize(const or_model *m, const double *a, double *b1, double *b2, double *flux)
{
  built_model bm;
  int status = build_model(m, &bm);
  if (status != OR_OK)
    return status;
  status = finalize_built(&bm, a, b1, b2, flux);
  built_free(&bm);
  return status;
}

/* ------------------------------------------------------------------------- */
/* Newton driver                                                              */
/* ------------------------------------------------------------------------- */

/* nonlinear_model.cpp:166-174 */
static double newton_linear_tolerance(const or_options *o, int adaptive, double prev)
{
  const double exact = o->linear_relative_tolerance;
  if (!adaptive || !isfinite(prev) || prev <= 100.0 * o->relative_tolerance || !(exact > 0.0) ||
      !isfinite(exact))
    return exact;
  const double loose = 1e-8 * fmin(1.0, prev);
  return exact > loose ? exact : loose;
}

static void expand(const or_system *s, const double *x, double *cand)
{
  for (int node = 0; node < s->N; ++node) {
    const int row = s->node_to_free[node];
    cand[node] = row >= 0 ? (double)s->node_sign[node] * x[row] : s->boundary[node];
  }
}

/* SolveSafeguarded: nonlinear_solver.cu:534-659 */
static void solve_safeguarded(const built_model *bm, const double *currents, const or_options *o,
                              double *state, or_info *info)
{
  const or_model *m = bm->m;
  const int N = m->node_count;
  info->status = OR_INVALID_ARGUMENT;
  info->iterations = 0;
  info->residual_l2 = INFINITY;
  info->linear_iterations = 0;
  info->verified_equation_residual_relative = INFINITY;
  for (int i = 0; i < N; ++i)
    state[i] = 0.0;
  for (int i = 0; i < m->dir_count; ++i)
    state[m->dir_nodes[i]] = m->dir_values[i];
  or_system *as = NULL;
  int status = assemble_built(bm, state, currents, 1, &as);
  if (status != OR_OK) {
    info->status = status;
    return;
  }
  {
    double *fs = malloc(sizeof(double) * (size_t)as->rows);
    for (int r = 0; r < as->rows; ++r)
      fs[r] = state[as->free_nodes[r]];
    expand(as, fs, state);
    free(fs);
  }
  or_system_free(as);
  as = NULL;
  status = assemble_built(bm, state, currents, 1, &as);
  if (status != OR_OK) {
    info->status = status;
    return;
  }
#define EQ_NORM(S, A, OUT)                                                                         \
  do {                                                                                             \
    double nrm = 0.0;                                                                              \
    for (int row = 0; row < (S)->rows; ++row) {                                                    \
      double v = -(S)->rhs_per_amp[row] - (S)->rhs_offset[row];                                    \
      for (int k = (S)->off[row]; k < (S)->off[row + 1]; ++k)                                      \
        v += (S)->val[k] * (A)[(S)->free_nodes[(S)->col[k]]];                                      \
      nrm = hypot(nrm, v);                                                                         \
    }                                                                                              \
    (OUT) = nrm;                                                                                   \
  } while (0)
  double norm;
  EQ_NORM(as, state, norm);
  const double scale = fmax(norm, DBL_MIN);
  const double eq_tol = o->relative_tolerance, step_tol = 100.0 * o->relative_tolerance;
  const int R = as->rows;
  double *rhs = malloc(sizeof(double) * (size_t)R), *x = malloc(sizeof(double) * (size_t)R);
  double *cand = malloc(sizeof(double) * (size_t)N), *trial = malloc(sizeof(double) * (size_t)N);
  info->status = OR_NONLINEAR_NOT_CONVERGED;
  for (int it = 0; it < o->max_newton_iterations; ++it) {
    if (!isfinite(norm)) {
      info->status = OR_NONFINITE;
      break;
    }
    for (int r = 0; r < R; ++r)
      rhs[r] = as->rhs_per_amp[r] + as->rhs_offset[r];
    int32_t lit = 0;
    double lres = 0.0;
    const int ls = or_pcg(R, as->off, as->col, as->val, as->diag, rhs, o->linear_relative_tolerance,
                          o->max_linear_iterations, x, &lit, &lres);
    info->linear_iterations += lit;
    info->last_linear_tolerance = o->linear_relative_tolerance;
    if (ls != OR_OK) {
      info->status = ls;
      info->iterations = lit;
      info->residual_l2 = lres;
      break;
    }
    expand(as, x, cand);
    double sn = 0.0, cn = 0.0;
    for (int i = 0; i < N; ++i) {
      sn = hypot(sn, cand[i] - state[i]);
      cn = hypot(cn, cand[i]);
    }
    const double rel = sn / fmax(cn, DBL_MIN);
    info->iterations = it + 1;
    info->residual_l2 = rel;
    if (!isfinite(rel)) {
      info->status = OR_NONFINITE;
      break;
    }
    if (rel < step_tol && norm / scale <= eq_tol) {
      info->status = OR_OK;
      break;
    }
    int accepted = 0;
    double alpha = 1.0;
    for (int bt = 0; bt < 20; ++bt, alpha *= 0.5) {
      for (int i = 0; i < N; ++i)
        trial[i] = state[i] + alpha * (cand[i] - state[i]);
      or_system *ts = NULL;
      status = assemble_built(bm, trial, currents, 1, &ts);
      if (status != OR_OK) {
        info->status = status;
        break;
      }
      double tn;
      EQ_NORM(ts, trial, tn);
      if (isfinite(tn) && (tn <= (1.0 - 1e-4 * alpha) * norm || tn / scale <= eq_tol)) {
        memcpy(state, trial, sizeof(double) * (size_t)N);
        or_system_free(as);
        as = ts;
        norm = tn;
        accepted = 1;
        break;
      }
      or_system_free(ts);
    }
    if (!accepted)
      break;
  }
#undef EQ_NORM
  info->verified_equation_residual_relative = norm / scale;
  or_system_free(as);
  free(rhs); free(x); free(cand); free(trial);
}

int or_solve_batch(const or_model *m, int32_t k, const double *currents, const double *warm,
                   const or_options *o, double *a, double *b1, double *b2, double *flux,
                   or_info *info)
{
  built_model bm;
  int status = build_model(m, &bm);
  for (int it = 0; it < k; ++it) {
    memset(&info[it], 0, sizeof(or_info));
    info[it].status = status != OR_OK ? status : OR_INVALID_ARGUMENT;
    info[it].residual_l2 = INFINITY;
    info[it].last_linear_tolerance = NAN;
    info[it].verified_equation_residual_relative = INFINITY;
  }
  if (status != OR_OK)
    return status;
  const int N = m->node_count, C = m->circuit_count, E = m->tri_count, R = bm.free_count;
  if (k <= 0 || !(o->relative_tolerance > 0.0) || !isfinite(o->relative_tolerance) ||
      o->max_newton_iterations < 0) {
    built_free(&bm);
    return OR_INVALID_ARGUMENT;
  }
  const int adaptive = o->adaptive_linear_tolerance && bm.has_nonlinear;
  double *relax = malloc(sizeof(double) * (size_t)k), *prev = malloc(sizeof(double) * (size_t)k);
  char *active = malloc((size_t)k), *done_ok = calloc((size_t)k, 1);
  double *x = malloc(sizeof(double) * (size_t)R), *cand = malloc(sizeof(double) * (size_t)N);
  double *rhs = malloc(sizeof(double) * (size_t)R);
  or_system **sys = calloc((size_t)k, sizeof(or_system *));
  for (int it = 0; it < k; ++it) {
    relax[it] = 1.0;
    prev[it] = INFINITY;
    active[it] = 1;
    double *st = a + (size_t)it * N;
    int finite = 1;
    for (int c = 0; c < C; ++c)
      if (!isfinite(currents[(size_t)it * C + c]))
        finite = 0;
    if (!finite) {
      active[it] = 0;
      continue;
    }
    for (int i = 0; i < N; ++i)
      st[i] = warm ? warm[(size_t)it * N + i] : 0.0;
    for (int i = 0; i < m->dir_count; ++i)
      st[m->dir_nodes[i]] = m->dir_values[i];
    if (!warm)
      for (int i = 0; i < N; ++i)
        if (bm.boundary[i] != 0.0)
          st[i] = bm.boundary[i];
  }
  for (int iter = 0; iter < o->max_newton_iterations; ++iter) {
    int any = 0;
    double tol = INFINITY;
    for (int it = 0; it < k; ++it)
      if (active[it]) {
        any = 1;
        const double t = newton_linear_tolerance(o, adaptive, prev[it]);
        tol = t < tol ? t : tol;
      }
    if (!any)
      break;
    for (int it = 0; it < k; ++it) {
      if (!active[it])
        continue;
      const int use_newton = (warm != NULL) || iter > 0;
      or_system *s = NULL;
      const int as =
          assemble_built(&bm, a + (size_t)it * N, currents + (size_t)it * C, use_newton, &s);
      if (as != OR_OK) {
        info[it].status = as;
        active[it] = 0;
        continue;
      }
      for (int r = 0; r < R; ++r)
        rhs[r] = s->rhs_per_amp[r] + s->rhs_offset[r];
      int32_t lit = 0;
      double lres = 0.0;
      const int ls = or_pcg(R, s->off, s->col, s->val, s->diag, rhs, tol, o->max_linear_iterations,
                            x, &lit, &lres);
      info[it].linear_iterations += lit;
      info[it].last_linear_tolerance = tol;
      if (ls != OR_OK) {
        info[it].status = ls;
        info[it].iterations = lit;
        info[it].residual_l2 = lres;
        active[it] = 0;
        or_system_free(s);
        continue;
      }
      expand(s, x, cand);
      or_system_free(s);
      double *st = a + (size_t)it * N;
      double dsq = 0.0, csq = 0.0;
      for (int i = 0; i < N; ++i) {
        const double d = cand[i] - st[i];
        dsq += d * d;
        csq += cand[i] * cand[i];
      }
      const double res = sqrt(dsq) / fmax(sqrt(csq), DBL_MIN);
      info[it].iterations = iter + 1;
      info[it].residual_l2 = res;
      if (!isfinite(res)) {
        info[it].status = OR_NONFINITE;
        active[it] = 0;
        continue;
      }
      if (iter > 5) {
        if (res > prev[it] && relax[it] > 0.125)
          relax[it] *= 0.5;
        else
          relax[it] += 0.1 * (1.0 - relax[it]);
      }
      for (int i = 0; i < N; ++i)
        st[i] += relax[it] * (cand[i] - st[i]);
      if (iter > 0 && res < 100.0 * o->relative_tolerance && tol <= o->linear_relative_tolerance) {
        info[it].status = OR_OK;
        active[it] = 0;
        done_ok[it] = 1;
      } else {
        prev[it] = res;
      }
    }
  }
  for (int it = 0; it < k; ++it) {
    if (active[it])
      info[it].status = OR_NONLINEAR_NOT_CONVERGED;
    if (info[it].status == OR_NONLINEAR_NOT_CONVERGED && o->recover_nonconvergence &&
        o->max_newton_iterations > 0) {
      or_info rec;
      memset(&rec, 0, sizeof(rec));
      solve_safeguarded(&bm, currents + (size_t)it * C, o, a + (size_t)it * N, &rec);
      rec.iterations += info[it].iterations;
      rec.linear_iterations += info[it].linear_iterations;
      info[it] = rec;
    }
    if (info[it].status == OR_OK || info[it].status == OR_NONLINEAR_NOT_CONVERGED) {
      const int fs = finalize_built(&bm, a + (size_t)it * N, b1 + (size_t)it * E,
                                    b2 + (size_t)it * E, flux + (size_t)it * C);
      if (fs != OR_OK)
        info[it].status = fs;
    }
  }
  free(relax); free(prev); free(active); free(done_ok); free(x); free(cand); free(rhs); free(sys);
  built_free(&bm);
  return OR_OK;
}
