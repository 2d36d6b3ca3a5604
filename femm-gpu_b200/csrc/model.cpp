// model.cpp -- host model checks, FEMM DC B-H spline, signed DOF folding and the
// topology of the device assembly plan.
#include "model.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace fg
{

const char *StatusName(Status status)
{
  switch (status) {
  case Status::kOk: return "OK";
  case Status::kInputIo: return "INPUT_IO";
  case Status::kInvalidArgument: return "INVALID_ARGUMENT";
  case Status::kUnsupportedFeature: return "UNSUPPORTED_FEATURE";
  case Status::kMeshInvalid: return "MESH_INVALID";
  case Status::kBoundaryInvalid: return "BOUNDARY_INVALID";
  case Status::kGpuUnavailable: return "GPU_UNAVAILABLE";
  case Status::kGpuAllocationFailed: return "GPU_ALLOCATION_FAILED";
  case Status::kAssemblyFailed: return "ASSEMBLY_FAILED";
  case Status::kLinearSolveNotConverged: return "LINEAR_SOLVE_NOT_CONVERGED";
  case Status::kLinearSolveBreakdown: return "LINEAR_SOLVE_BREAKDOWN";
  case Status::kNumericalNonfinite: return "NUMERICAL_NONFINITE";
  case Status::kOutputIo: return "OUTPUT_IO";
  case Status::kInternalError: return "INTERNAL_ERROR";
  case Status::kNonlinearSolveNotConverged: return "NONLINEAR_SOLVE_NOT_CONVERGED";
  case Status::kInvalidMaterial: return "INVALID_MATERIAL";
  }
  return "INTERNAL_ERROR";
}

namespace
{

// Slopes of FEMM's DC natural cubic (the tridiagonal "GetSlopes" system): Gaussian
// elimination with partial pivoting restricted to the band.  Every skipped update of
// the dense elimination subtracts an exact zero, so the result is the dense result.
bool SplineSlopes(const std::vector<double> &b, const std::vector<double> &h,
                  std::vector<double> *slope)
{
  const int n = static_cast<int>(b.size());
  std::vector<double> sub(n, 0.0), dia(n, 0.0), sup(n, 0.0), sup2(n, 0.0), rhs(n, 0.0);
  const double h0 = b[1] - b[0];
  dia[0] = 4.0 / h0;
  sup[0] = 2.0 / h0;
  rhs[0] = 6.0 * (h[1] - h[0]) / (h0 * h0);
  const double hl = b[n - 1] - b[n - 2];
  dia[n - 1] = 4.0 / hl;
  sub[n - 1] = 2.0 / hl;
  rhs[n - 1] = 6.0 * (h[n - 1] - h[n - 2]) / (hl * hl);
  for (int i = 1; i + 1 < n; ++i) {
    const double l = b[i] - b[i - 1], r = b[i + 1] - b[i];
    sub[i] = 2.0 / l;
    dia[i] = 4.0 * (l + r) / (l * r);
    sup[i] = 2.0 / r;
    rhs[i] = 6.0 * (h[i] - h[i - 1]) / (l * l) + 6.0 * (h[i + 1] - h[i]) / (r * r);
  }
  for (int k = 0; k < n; ++k) {
    if (k + 1 < n && std::abs(sub[k + 1]) > std::abs(dia[k])) {
      std::swap(dia[k], sub[k + 1]);
      std::swap(sup[k], dia[k + 1]);
      std::swap(sup2[k], sup[k + 1]);
      std::swap(rhs[k], rhs[k + 1]);
    }
    if (!(std::abs(dia[k]) > 0.0))
      return false;
    if (k + 1 < n) {
      const double f = sub[k + 1] / dia[k];
      sub[k + 1] -= f * dia[k];
      dia[k + 1] -= f * sup[k];
      sup[k + 1] -= f * sup2[k];
      rhs[k + 1] -= f * rhs[k];
    }
  }
  slope->assign(n, 0.0);
  for (int k = n - 1; k >= 0; --k) {
    double v = rhs[k];
    if (k + 1 < n)
      v -= sup[k] * (*slope)[k + 1];
    if (k + 2 < n)
      v -= sup2[k] * (*slope)[k + 2];
    (*slope)[k] = v / dia[k];
    if (!std::isfinite((*slope)[k]))
      return false;
  }
  return true;
}

// A segment's Hermite derivative has a root inside it: the curve is not monotone there.
bool SegmentHasInteriorExtremum(double length, double d0, double d1, double h0, double h1)
{
  const double c0 = d0;
  const double c1 = -2.0 * (2.0 * d0 * length + d1 * length + 3.0 * h0 - 3.0 * h1) / (length * length);
  const double c2 = 3.0 * (d0 * length + d1 * length + 2.0 * h0 - 2.0 * h1) / (length * length * length);
  double r0 = -1.0, r1 = -1.0;
  const double disc = c1 * c1 - 4.0 * c0 * c2;
  if (c2 == 0.0) {
    if (c1 != 0.0)
      r0 = -c0 / c1;
  } else if (disc > 0.0) {
    const double s = std::sqrt(disc);
    r0 = -(c1 + s) / (2.0 * c2);
    r1 = (-c1 + s) / (2.0 * c2);
  }
  return (r0 >= 0.0 && r0 <= length) || (r1 >= 0.0 && r1 <= length);
}

} // namespace

bool BuildBhSpline(BhCurve *curve)
{
  const size_t n = curve->b.size();
  if (n < 2 || curve->h.size() != n || curve->b[0] != 0.0 || curve->h[0] != 0.0)
    return false;
  if (!(curve->cold_secant > 0.0))
    curve->cold_secant = curve->h[1] / curve->b[1];
  for (;;) {
    for (size_t i = 1; i < n; ++i)
      if (!(curve->b[i] > curve->b[i - 1]) || curve->h[i] < 0.0 || !std::isfinite(curve->b[i]) ||
          !std::isfinite(curve->h[i]))
        return false;
    if (!SplineSlopes(curve->b, curve->h, &curve->slope))
      return false;
    bool monotone = true;
    for (size_t i = 1; i < n && monotone; ++i)
      monotone = !SegmentHasInteriorExtremum(curve->b[i] - curve->b[i - 1], curve->slope[i - 1],
                                             curve->slope[i], curve->h[i - 1], curve->h[i]);
    if (monotone)
      return true;
    if (++curve->smoothing_passes > 1024)
      return false;
    std::vector<double> nb = curve->b, nh = curve->h;
    for (size_t i = 1; i + 1 < n; ++i) {
      nb[i] = (curve->b[i - 1] + curve->b[i] + curve->b[i + 1]) / 3.0;
      nh[i] = (curve->h[i - 1] + curve->h[i] + curve->h[i + 1]) / 3.0;
    }
    curve->b.swap(nb);
    curve->h.swap(nh);
  }
}

void EvaluateBh(const BhCurve &c, double field_b, double out[4])
{
  const double b = std::abs(field_b);
  const size_t n = c.b.size();
  if (b == 0.0) {
    out[0] = 0.0;
    out[1] = c.slope[0];
    out[2] = c.slope[0];
    out[3] = 0.0;
    return;
  }
  double h = 0.0, dh = 0.0;
  if (b > c.b[n - 1]) {
    h = c.h[n - 1] + c.slope[n - 1] * (b - c.b[n - 1]);
    dh = c.slope[n - 1];
  } else {
    // First segment whose upper knot is >= b (the reference's linear scan order).
    const size_t k = static_cast<size_t>(std::lower_bound(c.b.begin() + 1, c.b.end(), b) - c.b.begin());
    if (k >= 1 && k < n) {
      const size_t i = k - 1;
      const double len = c.b[i + 1] - c.b[i];
      const double z = (b - c.b[i]) / len, z2 = z * z;
      h = (1.0 - 3.0 * z2 + 2.0 * z2 * z) * c.h[i] + z * (1.0 - 2.0 * z + z2) * len * c.slope[i] +
          z2 * (3.0 - 2.0 * z) * c.h[i + 1] + z2 * (z - 1.0) * len * c.slope[i + 1];
      dh = 6.0 * z * (z - 1.0) * c.h[i] / len + (1.0 - 4.0 * z + 3.0 * z2) * c.slope[i] +
           6.0 * z * (1.0 - z) * c.h[i + 1] / len + z * (3.0 * z - 2.0) * c.slope[i + 1];
    }
  }
  out[0] = h;
  out[1] = dh;
  out[2] = h / b;
  out[3] = 0.5 * (dh / (b * b) - h / (b * b * b));
}

bool ElementTerms(const double *p0, const double *p1, const double *p2, double *area,
                  double bx[3], double by[3])
{
  const double det = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
  if (!(det > 0.0) || !std::isfinite(det))
    return false;
  *area = 0.5 * det;
  const double dx[3] = {p1[1] - p2[1], p2[1] - p0[1], p0[1] - p1[1]};
  const double dy[3] = {p2[0] - p1[0], p0[0] - p2[0], p1[0] - p0[0]};
  for (int i = 0; i < 3; ++i) {
    bx[i] = dy[i] / det;
    by[i] = -dx[i] / det;
  }
  return true;
}

namespace
{
// Axisymmetric element validity (axisymmetric_p1.h:26-77): positive area and every
// seven-point quadrature radius strictly positive.
bool AxisymmetricValid(const double r[3], const double z[3])
{
  static const double bary[7][3] = {
      {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0},
      {0.059715871789770, 0.470142064105115, 0.470142064105115},
      {0.470142064105115, 0.059715871789770, 0.470142064105115},
      {0.470142064105115, 0.470142064105115, 0.059715871789770},
      {0.797426985353087, 0.101286507323456, 0.101286507323456},
      {0.101286507323456, 0.797426985353087, 0.101286507323456},
      {0.101286507323456, 0.101286507323456, 0.797426985353087}};
  const double det = (r[1] - r[0]) * (z[2] - z[0]) - (r[2] - r[0]) * (z[1] - z[0]);
  if (!(det > 0.0) || !std::isfinite(det))
    return false;
  for (int p = 0; p < 7; ++p) {
    double rp = 0.0;
    for (int l = 0; l < 3; ++l)
      rp += bary[p][l] * r[l];
    if (!(rp > 0.0) || !std::isfinite(rp))
      return false;
  }
  return true;
}
} // namespace

Status ValidateModel(const HostModel &m)
{
  const int32_t N = m.nodes(), E = m.triangles();
  if (N <= 0 || E <= 0 || m.materials.empty() ||
      (m.problem_type == 0 && (!(m.depth_m > 0.0) || !std::isfinite(m.depth_m))) ||
      m.circuit_count < 0 || m.dir_nodes.empty() || m.dir_nodes.size() != m.dir_values.size() ||
      m.tri.size() != static_cast<size_t>(3) * E)
    return Status::kInvalidArgument;
  std::vector<char> boundary(N, 0);
  for (size_t i = 0; i < m.dir_nodes.size(); ++i) {
    const int32_t node = m.dir_nodes[i];
    if (node < 0 || node >= N || boundary[node] || !std::isfinite(m.dir_values[i]))
      return Status::kBoundaryInvalid;
    boundary[node] = 1;
  }
  if (static_cast<int32_t>(m.dir_nodes.size()) == N)
    return Status::kBoundaryInvalid;
  for (int32_t i = 0; i < N; ++i)
    if (!std::isfinite(m.xy[2 * i]) || !std::isfinite(m.xy[2 * i + 1]) ||
        (m.problem_type == 1 && m.xy[2 * i] < 0.0))
      return Status::kMeshInvalid;
  for (const Material &mt : m.materials) {
    if (!(mt.nu0 > 0.0) || mt.alpha < 0.0 || !std::isfinite(mt.nu0) || !std::isfinite(mt.alpha) ||
        !std::isfinite(mt.j_per_a) || !std::isfinite(mt.hc) || !std::isfinite(mt.deg))
      return Status::kInvalidMaterial;
    if (mt.circuit < -1 || mt.circuit >= m.circuit_count || (mt.j_per_a != 0.0 && mt.circuit < 0))
      return Status::kInvalidMaterial;
    if (mt.curve < -1 || (mt.curve >= 0 && static_cast<size_t>(mt.curve) >= m.curves.size()))
      return Status::kInvalidMaterial;
    if (mt.curve >= 0) {
      const BhCurve &c = m.curves[mt.curve];
      if (c.b.size() < 2 || c.h.size() != c.b.size() || c.slope.size() != c.b.size() ||
          !(c.cold_secant > 0.0))
        return Status::kInvalidMaterial;
    }
  }
  for (int32_t e = 0; e < E; ++e) {
    if (m.tri_mat[e] < 0 || static_cast<size_t>(m.tri_mat[e]) >= m.materials.size())
      return Status::kInvalidMaterial;
    for (int l = 0; l < 3; ++l)
      if (m.tri[3 * e + l] < 0 || m.tri[3 * e + l] >= N)
        return Status::kMeshInvalid;
    const double *p0 = &m.xy[2 * m.tri[3 * e]], *p1 = &m.xy[2 * m.tri[3 * e + 1]],
                 *p2 = &m.xy[2 * m.tri[3 * e + 2]];
    double area, bx[3], by[3];
    if (!ElementTerms(p0, p1, p2, &area, bx, by))
      return Status::kMeshInvalid;
  }
  for (const AirGap &g : m.ages) {
    if (m.problem_type != 0)
      return Status::kUnsupportedFeature;
    if (g.points() < 3 || g.weight.size() != g.node.size() || g.node.size() % 4 != 0 || !(g.ri > 0.0) ||
        !(g.ro > g.ri) || !(g.arc_deg > 0.0) || !std::isfinite(g.cx) || !std::isfinite(g.cy) ||
        !std::isfinite(g.inner_shift) || !std::isfinite(g.outer_shift))
      return Status::kMeshInvalid;
    for (size_t l = 0; l < g.node.size(); ++l)
      if (g.node[l] < 0 || g.node[l] >= N || !std::isfinite(g.weight[l]))
        return Status::kMeshInvalid;
    const double dt = g.arc_deg / static_cast<double>(g.arcs());
    if (!(dt > 0.0) || !std::isfinite(dt))
      return Status::kMeshInvalid;
  }
  SignedDofs dofs;
  if (BuildSignedDofs(m, &dofs) != 0 || dofs.free_roots.empty())
    return Status::kBoundaryInvalid;
  if (m.problem_type == 1) {
    double scale = 1e-3;
    for (int32_t i = 0; i < N; ++i)
      scale = std::max(scale, m.xy[2 * i]);
    const double tol = 1e-12 * scale;
    for (int32_t i = 0; i < N; ++i)
      if (m.xy[2 * i] <= tol && (dofs.node_to_free[i] >= 0 || dofs.boundary[i] != 0.0))
        return Status::kBoundaryInvalid;
  }
  return Status::kOk;
}

int BuildSignedDofs(const HostModel &m, SignedDofs *out)
{
  const int32_t N = m.nodes();
  const size_t nc = m.con_a.size();
  if (N <= 0 || m.dir_nodes.size() != m.dir_values.size() || m.con_b.size() != nc ||
      m.con_sign.size() != nc)
    return 3;
  std::vector<int32_t> start(N + 1, 0);
  for (size_t i = 0; i < nc; ++i) {
    const int32_t a = m.con_a[i], b = m.con_b[i];
    if (a < 0 || b < 0 || a >= N || b >= N || (m.con_sign[i] != 1 && m.con_sign[i] != -1))
      return 1;
    if (a == b)
      return m.con_sign[i] < 0 ? 2 : 1;
    ++start[a + 1];
    ++start[b + 1];
  }
  for (int32_t i = 0; i < N; ++i)
    start[i + 1] += start[i];
  std::vector<int32_t> nbr(start[N]), fill(start.begin(), start.end() - 1);
  std::vector<int8_t> nbs(start[N]);
  for (size_t i = 0; i < nc; ++i) {
    nbr[fill[m.con_a[i]]] = m.con_b[i];
    nbs[fill[m.con_a[i]]++] = m.con_sign[i];
    nbr[fill[m.con_b[i]]] = m.con_a[i];
    nbs[fill[m.con_b[i]]++] = m.con_sign[i];
  }
  SignedDofs d;
  d.node_root.assign(N, -1);
  d.node_sign.assign(N, 0);
  std::vector<int32_t> stack;
  for (int32_t s = 0; s < N; ++s) {
    if (d.node_root[s] >= 0)
      continue;
    d.node_root[s] = s;
    d.node_sign[s] = 1;
    stack.assign(1, s);
    while (!stack.empty()) {
      const int32_t v = stack.back();
      stack.pop_back();
      for (int32_t k = start[v]; k < start[v + 1]; ++k) {
        const int32_t w = nbr[k];
        const int8_t sg = static_cast<int8_t>(d.node_sign[v] * nbs[k]);
        if (d.node_root[w] < 0) {
          d.node_root[w] = s;
          d.node_sign[w] = sg;
          stack.push_back(w);
        } else if (d.node_root[w] != s || d.node_sign[w] != sg) {
          return 2;
        }
      }
    }
  }
  std::vector<char> fixed(N, 0);
  std::vector<double> root_value(N, 0.0);
  for (size_t i = 0; i < m.dir_nodes.size(); ++i) {
    const int32_t node = m.dir_nodes[i];
    const double value = m.dir_values[i];
    if (node < 0 || node >= N || !std::isfinite(value))
      return 3;
    const int32_t root = d.node_root[node];
    const double rv = static_cast<double>(d.node_sign[node]) * value;
    if (fixed[root] && root_value[root] != rv)
      return 3;
    fixed[root] = 1;
    root_value[root] = rv;
  }
  std::vector<int32_t> root_to_free(N, -1);
  for (int32_t i = 0; i < N; ++i)
    if (d.node_root[i] == i && !fixed[i]) {
      root_to_free[i] = static_cast<int32_t>(d.free_roots.size());
      d.free_roots.push_back(i);
    }
  d.node_to_free.assign(N, -1);
  d.boundary.assign(N, 0.0);
  for (int32_t i = 0; i < N; ++i) {
    const int32_t root = d.node_root[i];
    d.node_to_free[i] = root_to_free[root];
    if (fixed[root])
      d.boundary[i] = static_cast<double>(d.node_sign[i]) * root_value[root];
  }
  *out = std::move(d);
  return 0;
}

Status BuildHostPlan(const HostModel &m, HostPlan *plan)
{
  HostPlan p;
  const Status valid = ValidateModel(m);
  if (valid != Status::kOk)
    return valid;
  p.problem_type = m.problem_type;
  p.N = m.nodes();
  p.E = m.triangles();
  p.C = m.circuit_count;
  if (BuildSignedDofs(m, &p.dofs) != 0)
    return Status::kBoundaryInvalid;
  const std::vector<int32_t> &n2f = p.dofs.node_to_free;
  const std::vector<int8_t> &sgn = p.dofs.node_sign;
  p.n = static_cast<int32_t>(p.dofs.free_roots.size());
  const int32_t n = p.n, E = p.E, N = p.N;
  if (n <= 0)
    return Status::kBoundaryInvalid;

  // Symbolic CSR: every (free row, free column) couple of a triangle, columns sorted.
  std::vector<int32_t> cand_off(n + 1, 0);
  for (int32_t e = 0; e < E; ++e)
    for (int i = 0; i < 3; ++i) {
      const int32_t r = n2f[m.tri[3 * e + i]];
      if (r < 0)
        continue;
      for (int j = 0; j < 3; ++j)
        if (n2f[m.tri[3 * e + j]] >= 0)
          ++cand_off[r + 1];
    }
  // Air-gap couples: every (free, free) pair of each arc's ten-node stencil.
  auto for_each_age_entry = [&m](auto &&visit) {
    for (const AirGap &g : m.ages)
      for (int32_t k = 0; k < g.arcs(); ++k) {
        int32_t node[10];
        double weight[10];
        AirGapStencil(g, k, node, weight);
        for (int i = 0; i < 10; ++i)
          for (int j = 0; j < 10; ++j)
            visit(g, k, i, j, node, weight);
      }
  };
  for_each_age_entry([&](const AirGap &, int32_t, int i, int j, const int32_t *node, const double *) {
    const int32_t r = n2f[node[i]];
    if (r >= 0 && n2f[node[j]] >= 0)
      ++cand_off[r + 1];
  });
  for (int32_t r = 0; r < n; ++r)
    cand_off[r + 1] += cand_off[r];
  std::vector<int32_t> cand(cand_off[n]), cfill(cand_off.begin(), cand_off.end() - 1);
  for (int32_t e = 0; e < E; ++e)
    for (int i = 0; i < 3; ++i) {
      const int32_t r = n2f[m.tri[3 * e + i]];
      if (r < 0)
        continue;
      for (int j = 0; j < 3; ++j) {
        const int32_t c = n2f[m.tri[3 * e + j]];
        if (c >= 0)
          cand[cfill[r]++] = c;
      }
    }
  for_each_age_entry([&](const AirGap &, int32_t, int i, int j, const int32_t *node, const double *) {
    const int32_t r = n2f[node[i]], c = n2f[node[j]];
    if (r >= 0 && c >= 0)
      cand[cfill[r]++] = c;
  });
  p.row_offsets.assign(n + 1, 0);
  p.diag_slot.assign(n, -1);
  for (int32_t r = 0; r < n; ++r) {
    auto first = cand.begin() + cand_off[r], last = cand.begin() + cand_off[r + 1];
    std::sort(first, last);
    last = std::unique(first, last);
    p.row_offsets[r + 1] = p.row_offsets[r] + static_cast<int32_t>(last - first);
  }
  p.nnz = p.row_offsets[n];
  p.columns.resize(p.nnz);
  for (int32_t r = 0; r < n; ++r) {
    std::copy(cand.begin() + cand_off[r], cand.begin() + cand_off[r] + (p.row_offsets[r + 1] - p.row_offsets[r]),
              p.columns.begin() + p.row_offsets[r]);
    for (int32_t k = p.row_offsets[r]; k < p.row_offsets[r + 1]; ++k)
      if (p.columns[k] == r)
        p.diag_slot[r] = k;
    if (p.diag_slot[r] < 0)
      return Status::kAssemblyFailed;
  }
  std::vector<int32_t>().swap(cand);
  auto find_slot = [&p](int32_t r, int32_t c) {
    const auto b = p.columns.begin() + p.row_offsets[r], e = p.columns.begin() + p.row_offsets[r + 1];
    return static_cast<int32_t>(std::lower_bound(b, e, c) - p.columns.begin());
  };

  // Matrix contributors per slot, in element / i / j order.
  p.contrib_off.assign(p.nnz + 1, 0);
  for (int32_t e = 0; e < E; ++e)
    for (int i = 0; i < 3; ++i) {
      const int32_t r = n2f[m.tri[3 * e + i]];
      if (r < 0)
        continue;
      for (int j = 0; j < 3; ++j) {
        const int32_t c = n2f[m.tri[3 * e + j]];
        if (c >= 0)
          ++p.contrib_off[find_slot(r, c) + 1];
      }
    }
  for (int64_t s = 0; s < p.nnz; ++s)
    p.contrib_off[s + 1] += p.contrib_off[s];
  p.contrib.resize(p.contrib_off[p.nnz]);
  {
    std::vector<int32_t> fill(p.contrib_off.begin(), p.contrib_off.end() - 1);
    for (int32_t e = 0; e < E; ++e)
      for (int i = 0; i < 3; ++i) {
        const int32_t ni = m.tri[3 * e + i];
        const int32_t r = n2f[ni];
        if (r < 0)
          continue;
        for (int j = 0; j < 3; ++j) {
          const int32_t nj = m.tri[3 * e + j];
          const int32_t c = n2f[nj];
          if (c < 0)
            continue;
          const int negative = (sgn[ni] * sgn[nj]) < 0 ? 1 : 0;
          p.contrib[fill[find_slot(r, c)]++] = (e << 4) | (PairIndex(i, j) << 1) | negative;
        }
      }
  }

  // Element geometry, RHS contributors and the fixed permanent-magnet / coil loads.
  p.elem_nodes.assign(m.tri.begin(), m.tri.end());
  p.elem_mat.assign(m.tri_mat.begin(), m.tri_mat.end());
  const int geo_rows = m.problem_type == 0 ? 7 : 6;
  p.elem_geo.assign(static_cast<size_t>(geo_rows) * E, 0.0);
  p.rhs_off.assign(n + 1, 0);
  p.pm_rhs.assign(n, 0.0);
  p.circuit_rhs.assign(static_cast<size_t>(p.C) * n, 0.0);
  for (int32_t e = 0; e < E; ++e)
    for (int i = 0; i < 3; ++i) {
      const int32_t r = n2f[m.tri[3 * e + i]];
      if (r >= 0)
        ++p.rhs_off[r + 1];
    }
  for (int32_t r = 0; r < n; ++r)
    p.rhs_off[r + 1] += p.rhs_off[r];
  p.rhs_contrib.resize(p.rhs_off[n]);
  std::vector<int32_t> rfill(p.rhs_off.begin(), p.rhs_off.end() - 1);
  static const double bary[7][3] = {
      {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0},
      {0.059715871789770, 0.470142064105115, 0.470142064105115},
      {0.470142064105115, 0.059715871789770, 0.470142064105115},
      {0.470142064105115, 0.470142064105115, 0.059715871789770},
      {0.797426985353087, 0.101286507323456, 0.101286507323456},
      {0.101286507323456, 0.797426985353087, 0.101286507323456},
      {0.101286507323456, 0.101286507323456, 0.797426985353087}};
  static const double qw[7] = {0.225, 0.132394152788506, 0.132394152788506, 0.132394152788506,
                               0.125939180544827, 0.125939180544827, 0.125939180544827};
  for (int32_t e = 0; e < E; ++e) {
    const Material &mt = m.materials[m.tri_mat[e]];
    const int32_t *tn = &m.tri[3 * e];
    const double *p0 = &m.xy[2 * tn[0]], *p1 = &m.xy[2 * tn[1]], *p2 = &m.xy[2 * tn[2]];
    const double theta = mt.deg * kPi / 180.0;
    const double hcx = mt.hc * std::cos(theta), hcy = mt.hc * std::sin(theta);
    double pm[3] = {0, 0, 0}, coil[3] = {0, 0, 0};
    if (m.problem_type == 0) {
      double area, bx[3], by[3];
      ElementTerms(p0, p1, p2, &area, bx, by);
      p.elem_geo[e] = area;
      for (int l = 0; l < 3; ++l) {
        p.elem_geo[static_cast<size_t>(1 + l) * E + e] = bx[l];
        p.elem_geo[static_cast<size_t>(4 + l) * E + e] = by[l];
        pm[l] = 0.0 + area * (hcx * bx[l] + hcy * by[l]);
        coil[l] = 0.0 + area * mt.j_per_a * (1.0 / 3.0);
      }
    } else {
      const double r[3] = {p0[0], p1[0], p2[0]}, z[3] = {p0[1], p1[1], p2[1]};
      for (int l = 0; l < 3; ++l) {
        p.elem_geo[static_cast<size_t>(l) * E + e] = r[l];
        p.elem_geo[static_cast<size_t>(3 + l) * E + e] = z[l];
      }
      if (!AxisymmetricValid(r, z))
        return Status::kMeshInvalid;
      const double det = (r[1] - r[0]) * (z[2] - z[0]) - (r[2] - r[0]) * (z[1] - z[0]);
      const double dndr[3] = {(z[1] - z[2]) / det, (z[2] - z[0]) / det, (z[0] - z[1]) / det};
      const double dndz[3] = {(r[2] - r[1]) / det, (r[0] - r[2]) / det, (r[1] - r[0]) / det};
      const double area = 0.5 * det;
      for (int q = 0; q < 7; ++q) {
        double rq = 0.0;
        for (int l = 0; l < 3; ++l)
          rq += bary[q][l] * r[l];
        const double w = kTwoPi * rq * (area * qw[q]);
        for (int l = 0; l < 3; ++l) {
          const double br = -dndz[l], bz = dndr[l] + bary[q][l] / rq;
          pm[l] += w * (hcx * br + hcy * bz);
          coil[l] += w * mt.j_per_a * bary[q][l];
        }
      }
    }
    for (int i = 0; i < 3; ++i) {
      const int32_t r = n2f[tn[i]];
      if (r < 0)
        continue;
      p.rhs_contrib[rfill[r]++] = (e << 3) | (i << 1) | (sgn[tn[i]] < 0 ? 1 : 0);
      p.pm_rhs[r] += static_cast<double>(sgn[tn[i]]) * pm[i];
      if (mt.circuit >= 0)
        p.circuit_rhs[static_cast<size_t>(mt.circuit) * n + r] += static_cast<double>(sgn[tn[i]]) * coil[i];
    }
  }

  // Air-gap stiffness (relative-reluctivity element matrix times 1/mu0) and the load of
  // its fixed nodes, in band / arc / i / j order.
  if (!m.ages.empty()) {
    p.age_val.assign(p.nnz, 0.0);
    p.age_rhs.assign(n, 0.0);
    const std::vector<double> &fixed = p.dofs.boundary;
    double mg[10][10];
    const AirGap *current = nullptr;
    bool ok = true;
    for_each_age_entry([&](const AirGap &g, int32_t, int i, int j, const int32_t *node,
                           const double *weight) {
      if (current != &g) {
        const AirGapTerms t = AirGapBandTerms(g);
        ok = ok && AirGapElementMatrix(t.K, t.Ki, t.ci, t.co, mg);
        current = &g;
      }
      if (!ok)
        return;
      const double value = mg[i][j] * weight[i] * weight[j] * (1.0 / kMu0);
      const int32_t r = n2f[node[i]], c = n2f[node[j]];
      if (r >= 0 && c >= 0)
        p.age_val[find_slot(r, c)] += static_cast<double>(sgn[node[i]] * sgn[node[j]]) * value;
      else if (r >= 0)
        p.age_rhs[r] -= static_cast<double>(sgn[node[i]]) * value * fixed[node[j]];
    });
    if (!ok)
      return Status::kMeshInvalid;
  }

  // SELL-32 layout of the symbolic pattern.
  p.n_pad = (n + 31) / 32 * 32;
  p.slices = p.n_pad / 32;
  p.row_len.assign(p.n_pad, 0);
  p.slice_off.assign(p.slices + 1, 0);
  for (int32_t r = 0; r < n; ++r)
    p.row_len[r] = p.row_offsets[r + 1] - p.row_offsets[r];
  for (int32_t s = 0; s < p.slices; ++s) {
    int32_t w = 0;
    for (int32_t r = 32 * s; r < 32 * s + 32; ++r)
      w = std::max(w, p.row_len[r]);
    p.slice_off[s + 1] = p.slice_off[s] + 32 * w;
  }
  p.positions = p.slice_off[p.slices];
  p.sell_col.assign(p.positions, 0);
  for (int32_t r = 0; r < p.n_pad; ++r) {
    const int32_t s = r / 32, lane = r % 32;
    const int32_t width = (p.slice_off[s + 1] - p.slice_off[s]) / 32;
    for (int32_t w = 0; w < width; ++w)
      p.sell_col[p.slice_off[s] + 32 * w + lane] =
          (r < n && w < p.row_len[r]) ? p.columns[p.row_offsets[r] + w] : (r < n ? r : 0);
  }

  // Materials and curves.
  const size_t M = m.materials.size();
  p.mat_nu0.resize(M);
  p.mat_alpha.resize(M);
  p.mat_cold.resize(M);
  p.mat_jpa.resize(M);
  p.mat_curve_off.resize(M);
  p.mat_curve_cnt.resize(M);
  p.mat_circuit.resize(M);
  std::vector<int32_t> curve_start;
  for (const BhCurve &c : m.curves) {
    curve_start.push_back(static_cast<int32_t>(p.curve_b.size()));
    p.curve_b.insert(p.curve_b.end(), c.b.begin(), c.b.end());
    p.curve_h.insert(p.curve_h.end(), c.h.begin(), c.h.end());
    p.curve_slope.insert(p.curve_slope.end(), c.slope.begin(), c.slope.end());
  }
  if (p.curve_b.empty()) {
    p.curve_b.push_back(0.0);
    p.curve_h.push_back(0.0);
    p.curve_slope.push_back(0.0);
  }
  for (size_t i = 0; i < M; ++i) {
    const Material &mt = m.materials[i];
    p.mat_nu0[i] = mt.nu0;
    p.mat_alpha[i] = mt.alpha;
    p.mat_jpa[i] = mt.j_per_a;
    p.mat_circuit[i] = mt.circuit;
    p.mat_curve_off[i] = mt.curve >= 0 ? curve_start[mt.curve] : -1;
    p.mat_curve_cnt[i] = mt.curve >= 0 ? static_cast<int32_t>(m.curves[mt.curve].b.size()) : -1;
    p.mat_cold[i] = mt.curve >= 0 ? m.curves[mt.curve].cold_secant : 0.0;
    if (mt.curve >= 0 || mt.alpha != 0.0)
      p.has_nonlinear = true;
  }

  // Elements of each circuit, in element order, for flux recovery.
  p.circuit_elem_off.assign(p.C + 1, 0);
  for (int32_t e = 0; e < E; ++e) {
    const int32_t c = m.materials[m.tri_mat[e]].circuit;
    if (c >= 0)
      ++p.circuit_elem_off[c + 1];
  }
  for (int32_t c = 0; c < p.C; ++c)
    p.circuit_elem_off[c + 1] += p.circuit_elem_off[c];
  p.circuit_elems.resize(p.circuit_elem_off[p.C]);
  {
    std::vector<int32_t> fill(p.circuit_elem_off.begin(), p.circuit_elem_off.end() - 1);
    for (int32_t e = 0; e < E; ++e) {
      const int32_t c = m.materials[m.tri_mat[e]].circuit;
      if (c >= 0)
        p.circuit_elems[fill[c]++] = e;
    }
  }
  (void)N;
  *plan = std::move(p);
  return Status::kOk;
}

} // namespace fg
