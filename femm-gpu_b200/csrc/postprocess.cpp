// postprocess.cpp -- frozen-state postprocessing: weighted-stress force and torque on a
// selected region and FEMM-smoothed radial air-gap flux density samples.
//
// Follows ComputeFrozenPostprocess and its reusable plan (gpu_solver/src/postprocess/
// field_postprocess.cpp:205-403), FEMM's nodal B smoothing (:30-190) and the weighted-
// stress mask (weighted_stress.cu:24-193):
//
// * Mask: the scalar Laplace problem with per-element weight sqrt(area) (FEMM's default
//   WeightingScheme 0), fixed to 1 on the selected region's nodes and to 0 on other
//   non-air regions and on the Dirichlet nodes that are not symmetry apex nodes, periodic
//   across every node constraint (each pair taken with sign +1), solved by the library's
//   PCG on the GPU and thresholded at 0.5.
// * Force density from element B and the mask gradient h = curl(mask):
//     fx = ((Bx^2 - By^2) hx + 2 Bx By hy) / (2 mu0),  fy = (2 Bx By hx + (By^2 - Bx^2) hy) / (2 mu0),
//   summed over elements with weight area x depth in element order; torque about the
//   origin from the element centroids.
// * Air-gap samples: the first containing element (element order, bounding-box filtered)
//   of each probe on the circle, which must be air; FEMM's nodal B at its corners;
//   barycentric interpolation; the radial component.
//
// The host path keeps the reference's operation order, so it agrees with it bit for bit on
// the same mask and solution.  The device path (fg_postprocess_compute_device) sums per-CTA
// partials in a fixed order instead: deterministic, equal to the host path within rounding.
#include "postprocess.h"
#include "solver.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <vector>

namespace fg
{
namespace
{

struct Select {
  const fg_postprocess_options &o;
  const HostModel &m;
  bool selected(int32_t mat) const
  {
    return o.selected_group_number >= 0 ? m.materials[mat].group == o.selected_group_number
                                        : mat == o.selected_material_label;
  }
  bool air(int32_t mat) const
  {
    return o.air_group_number >= 0 ? m.materials[mat].group == o.air_group_number
                                   : mat == o.air_material_label;
  }
};

bool ValidOptions(const HostModel &m, const fg_postprocess_options &o)
{
  const int32_t M = static_cast<int32_t>(m.materials.size());
  return !((o.selected_group_number < 0 && (o.selected_material_label < 0 || o.selected_material_label >= M)) ||
           (o.air_group_number < 0 && (o.air_material_label < 0 || o.air_material_label >= M)) ||
           (o.selected_group_number >= 0 && o.selected_group_number == o.air_group_number) ||
           (o.selected_group_number < 0 && o.air_group_number < 0 &&
            o.selected_material_label == o.air_material_label) ||
           !(o.mask_relative_tolerance > 0.0) || !std::isfinite(o.mask_relative_tolerance) ||
           o.max_mask_iterations <= 0 || o.symmetry_apex_count < 0 ||
           (o.symmetry_apex_count > 0 && !o.symmetry_apex_nodes));
}

// FEMM's nodal B at the three corners of `element` (the DC subset of GetNodalB):
// inverse-centroid-distance averaging when every element around the corner has the
// element's label, else the interface traversal both ways around the corner, keeping Bt
// from the source-side element and Bn from A, with FEMM's sharp-corner fallback.  The
// accessors read a / b1 / b2 by global node / element id.
template <class A, class B1, class B2>
bool NodalB(const HostModel &m, const A &a, const B1 &b1, const B2 &b2,
            const std::vector<std::vector<int32_t>> &incident, int32_t element, double nbx[3],
            double nby[3])
{
  const int32_t *tri = m.tri.data();
  const double *xy = m.xy.data();
  const int32_t mat = m.tri_mat[element];
  for (int l = 0; l < 3; ++l) {
    const int32_t node = tri[3 * element + l];
    const std::vector<int32_t> &around = incident[node];
    bool same = true;
    for (int32_t e : around)
      same = same && m.tri_mat[e] == mat;
    nbx[l] = 0.0;
    nby[l] = 0.0;
    if (same) {
      double wsum = 0.0;
      for (int32_t e : around) {
        const int32_t *t = &tri[3 * e];
        const double cx = (xy[2 * t[0]] + xy[2 * t[1]] + xy[2 * t[2]]) / 3.0;
        const double cy = (xy[2 * t[0] + 1] + xy[2 * t[1] + 1] + xy[2 * t[2] + 1]) / 3.0;
        const double w = 1.0 / std::hypot(xy[2 * node] - cx, xy[2 * node + 1] - cy);
        if (!(w > 0.0) || !std::isfinite(w))
          return false;
        wsum += w;
        nbx[l] += w * b1(e);
        nby[l] += w * b2(e);
      }
      nbx[l] /= wsum;
      nby[l] /= wsum;
      continue;
    }
    auto position = [&](int32_t e) {
      for (int i = 0; i < 3; ++i)
        if (tri[3 * e + i] == node)
          return i;
      return -1;
    };
    auto across = [&](int32_t current, int32_t other) {
      for (int32_t e : around) {
        if (e == current)
          continue;
        for (int i = 0; i < 3; ++i)
          if (tri[3 * e + i] == other)
            return e;
      }
      return static_cast<int32_t>(-1);
    };
    double wsum = 0.0;
    double t1[2] = {0.0, 0.0}, t2[2] = {0.0, 0.0};
    bool edge_of_mesh = false;
    // Two sweeps around the corner: across the edge to the corner's previous node (local + 2),
    // then across the edge to its next node (local + 1); each stops at the first label change.
    for (int sweep = 0; sweep < 2 && !edge_of_mesh; ++sweep) {
      int32_t current = element;
      for (size_t step = 0; step < around.size(); ++step) {
        const int i = position(current);
        if (i < 0)
          return false;
        const int32_t other = tri[3 * current + (sweep == 0 ? (i + 2) % 3 : (i + 1) % 3)];
        const int32_t next = across(current, other);
        if (next < 0) {
          nbx[l] = b1(current);
          nby[l] = b2(current);
          edge_of_mesh = true;
          break;
        }
        if (m.tri_mat[next] != mat) {
          const double dx = xy[2 * other] - xy[2 * node], dy = xy[2 * other + 1] - xy[2 * node + 1];
          const double len = std::hypot(dx, dy);
          if (!(len > 0.0))
            return false;
          const double tx = dx / len, ty = dy / len;
          const double bt = b1(current) * tx + b2(current) * ty;
          const double bn = (a(other) - a(node)) / len;
          const double w = 0.5 / len;
          nbx[l] += w * (tx * bt + ty * bn);
          nby[l] += w * (ty * bt - tx * bn);
          wsum += w;
          const double len2 = std::hypot(xy[2 * other] - xy[2 * node], xy[2 * other + 1] - xy[2 * node + 1]);
          double *t = sweep == 0 ? t1 : t2;
          t[0] = (xy[2 * other] - xy[2 * node]) / len2;
          t[1] = (xy[2 * other + 1] - xy[2 * node + 1]) / len2;
          break;
        }
        current = next;
      }
    }
    if (edge_of_mesh)
      continue;
    if (!(wsum > 0.0))
      return false;
    nbx[l] /= wsum;
    nby[l] /= wsum;
    const bool simple = std::hypot(t1[0], t1[1]) < 0.9 || std::hypot(t2[0], t2[1]) < 0.9 ||
                        (-t1[0] * t2[0] - t1[1] * t2[1]) > 0.985;
    if (!simple) {
      double largest = 0.0;
      for (int32_t e : around)
        if (m.tri_mat[e] == mat)
          largest = std::max(largest, std::hypot(b1(e), b2(e)));
      const double own = std::hypot(b1(element), b2(element));
      nbx[l] = own > 0.0 ? largest * b1(element) / own : 0.0;
      nby[l] = own > 0.0 ? largest * b2(element) / own : 0.0;
    }
  }
  return true;
}

// Barycentric coordinates of (x, y) in triangle e (TriangleBarycentric,
// field_postprocess.cpp:14-28).
bool Barycentric(const HostModel &m, int32_t e, double x, double y, double lam[3])
{
  const double *p0 = &m.xy[2 * m.tri[3 * e]], *p1 = &m.xy[2 * m.tri[3 * e + 1]], *p2 = &m.xy[2 * m.tri[3 * e + 2]];
  const double det = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
  if (!(det > 0.0) || !std::isfinite(det))
    return false;
  lam[1] = ((x - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (y - p0[1])) / det;
  lam[2] = ((p1[0] - p0[0]) * (y - p0[1]) - (x - p0[0]) * (p1[1] - p0[1])) / det;
  lam[0] = 1.0 - lam[1] - lam[2];
  return std::isfinite(lam[0]) && std::isfinite(lam[1]) && std::isfinite(lam[2]);
}

} // namespace

Status WeightedStressMask(const HostModel &m, const fg_postprocess_options &o, std::vector<double> *mask)
{
  if (!ValidOptions(m, o))
    return Status::kInvalidArgument;
  const int32_t N = m.nodes(), E = m.triangles();
  const Select sel{o, m};
  std::map<std::pair<int32_t, int32_t>, std::vector<int32_t>> edges;
  bool seen = false;
  for (int32_t e = 0; e < E; ++e) {
    seen = seen || sel.selected(m.tri_mat[e]);
    for (int l = 0; l < 3; ++l) {
      const int32_t p = m.tri[3 * e + l], q = m.tri[3 * e + (l + 1) % 3];
      edges[{std::min(p, q), std::max(p, q)}].push_back(e);
    }
  }
  if (!seen)
    return Status::kInvalidMaterial;
  // FEMM's MakeMask rejects a selection that touches a non-air region.
  for (const auto &kv : edges) {
    bool s = false, other = false;
    for (int32_t e : kv.second) {
      const int32_t mat = m.tri_mat[e];
      s = s || sel.selected(mat);
      other = other || (!sel.selected(mat) && !sel.air(mat));
    }
    if (s && other)
      return Status::kInvalidMaterial;
  }
  std::vector<double> fixed(N, std::numeric_limits<double>::quiet_NaN());
  const int32_t *apex = o.symmetry_apex_nodes, *apex_end = apex + o.symmetry_apex_count;
  for (int32_t d : m.dir_nodes)
    if (std::find(apex, apex_end, d) == apex_end)
      fixed[d] = 0.0;
  for (int32_t e = 0; e < E; ++e) {
    const int32_t mat = m.tri_mat[e];
    if (sel.selected(mat)) {
      for (int l = 0; l < 3; ++l) {
        const int32_t v = m.tri[3 * e + l];
        if (std::isfinite(fixed[v]) && fixed[v] != 1.0)
          return Status::kBoundaryInvalid;
        fixed[v] = 1.0;
      }
    } else if (!sel.air(mat)) {
      for (int l = 0; l < 3; ++l) {
        const int32_t v = m.tri[3 * e + l];
        if (!std::isfinite(fixed[v]))
          fixed[v] = 0.0;
      }
    }
  }
  // Node stiffness, per row in ascending column order, accumulated in element order.
  std::vector<std::map<int32_t, double>> K(N);
  for (int32_t e = 0; e < E; ++e) {
    const int32_t *t = &m.tri[3 * e];
    double area, bx[3], by[3];
    if (!ElementTerms(&m.xy[2 * t[0]], &m.xy[2 * t[1]], &m.xy[2 * t[2]], &area, bx, by))
      return Status::kMeshInvalid;
    const double w = std::sqrt(area);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        double &k = K[t[r]][t[c]];
        k += w * area * (bx[r] * bx[c] + by[r] * by[c]);
        if (!std::isfinite(k))
          return Status::kNumericalNonfinite;
      }
  }
  if (std::all_of(fixed.begin(), fixed.end(), [](double v) { return std::isfinite(v); })) {
    mask->assign(N, 0.0);
    for (int32_t v = 0; v < N; ++v)
      (*mask)[v] = fixed[v] > 0.5 ? 1.0 : 0.0;
    return Status::kOk;
  }
  // The mask is periodic across the constraint pairs whatever their magnetic sign.
  HostModel mm;
  mm.xy = m.xy;
  mm.con_a = m.con_a;
  mm.con_b = m.con_b;
  mm.con_sign.assign(m.con_sign.size(), 1);
  for (int32_t v = 0; v < N; ++v)
    if (std::isfinite(fixed[v])) {
      mm.dir_nodes.push_back(v);
      mm.dir_values.push_back(fixed[v]);
    }
  SignedDofs dofs;
  if (BuildSignedDofs(mm, &dofs) != 0 || dofs.free_roots.empty())
    return Status::kBoundaryInvalid;
  const int32_t n = static_cast<int32_t>(dofs.free_roots.size());
  // Signed reduction (ReduceSignedSystem, nonlinear_model.cpp:321-394).
  std::vector<std::map<int32_t, double>> rows(n);
  std::vector<double> offset(n, 0.0);
  for (int32_t v = 0; v < N; ++v) {
    const int32_t r = dofs.node_to_free[v];
    if (r < 0)
      continue;
    const double rs = dofs.node_sign[v];
    for (const auto &kv : K[v]) {
      const int32_t c = dofs.node_to_free[kv.first];
      if (c < 0) {
        offset[r] -= rs * kv.second * dofs.boundary[kv.first];
      } else {
        double &k = rows[r][c];
        k += rs * static_cast<double>(dofs.node_sign[kv.first]) * kv.second;
        if (!std::isfinite(k))
          return Status::kNumericalNonfinite;
      }
    }
  }
  std::vector<int32_t> ro(n + 1, 0), col;
  std::vector<double> val, diag(n, 0.0), rhs(n);
  for (int32_t r = 0; r < n; ++r) {
    for (const auto &kv : rows[r]) {
      col.push_back(kv.first);
      val.push_back(kv.second);
      if (kv.first == r)
        diag[r] = kv.second;
    }
    ro[r + 1] = static_cast<int32_t>(col.size());
    rhs[r] = 0.0 + offset[r];
    if (!(diag[r] > 0.0) || !std::isfinite(diag[r]) || !std::isfinite(offset[r]))
      return Status::kAssemblyFailed;
  }
  std::vector<double> x(n, 0.0);
  fg_linear_info info{};
  const int st = fg_csr_pcg(n, ro.data(), col.data(), val.data(), 0, diag.data(), 1, rhs.data(),
                            o.mask_relative_tolerance, o.max_mask_iterations, x.data(), &info);
  if (st != 0)
    return static_cast<Status>(st);
  if (info.status != 0)
    return static_cast<Status>(info.status);
  // FEMM's WeightingScheme 0 thresholds every solved node at 0.5.
  mask->assign(N, 0.0);
  for (int32_t v = 0; v < N; ++v) {
    const int32_t r = dofs.node_to_free[v];
    const double value = r >= 0 ? dofs.node_sign[v] * x[r] : dofs.boundary[v];
    (*mask)[v] = value > 0.5 ? 1.0 : 0.0;
  }
  return Status::kOk;
}

namespace
{

// The recipe NodalB follows at corner l of `element` (same control flow, nothing read from
// a solution), appended to plan->corners and the term arrays.
void BuildCorner(const HostModel &m, int32_t element, int l, PostprocessPlan *plan)
{
  const int32_t *tri = m.tri.data();
  const double *xy = m.xy.data();
  const int32_t mat = m.tri_mat[element];
  const int32_t node = tri[3 * element + l];
  const std::vector<int32_t> &around = plan->incident[node];
  CornerStencil c{};
  c.first = static_cast<int32_t>(plan->term_elem.size());
  c.element = element;
  c.node = node;
  auto term = [&](int32_t e, int32_t other, double w, double tx, double ty, double len) {
    plan->term_elem.push_back(e);
    plan->term_node.push_back(other);
    plan->term_w.push_back(w);
    plan->term_tx.push_back(tx);
    plan->term_ty.push_back(ty);
    plan->term_len.push_back(len);
  };
  auto truncate = [&] {
    plan->term_elem.resize(c.first);
    plan->term_node.resize(c.first);
    plan->term_w.resize(c.first);
    plan->term_tx.resize(c.first);
    plan->term_ty.resize(c.first);
    plan->term_len.resize(c.first);
  };
  auto finish = [&](int kind) {
    c.kind = kind;
    c.count = static_cast<int32_t>(plan->term_elem.size()) - c.first;
    plan->corners.push_back(c);
  };
  bool same = true;
  for (int32_t e : around)
    same = same && m.tri_mat[e] == mat;
  if (same) {
    double wsum = 0.0;
    for (int32_t e : around) {
      const int32_t *t = &tri[3 * e];
      const double cx = (xy[2 * t[0]] + xy[2 * t[1]] + xy[2 * t[2]]) / 3.0;
      const double cy = (xy[2 * t[0] + 1] + xy[2 * t[1] + 1] + xy[2 * t[2] + 1]) / 3.0;
      const double w = 1.0 / std::hypot(xy[2 * node] - cx, xy[2 * node + 1] - cy);
      if (!(w > 0.0) || !std::isfinite(w))
        return finish(-1);
      wsum += w;
      term(e, -1, w, 0.0, 0.0, 0.0);
    }
    c.wsum = wsum;
    return finish(0);
  }
  auto position = [&](int32_t e) {
    for (int i = 0; i < 3; ++i)
      if (tri[3 * e + i] == node)
        return i;
    return -1;
  };
  auto across = [&](int32_t current, int32_t other) {
    for (int32_t e : around) {
      if (e == current)
        continue;
      for (int i = 0; i < 3; ++i)
        if (tri[3 * e + i] == other)
          return e;
    }
    return static_cast<int32_t>(-1);
  };
  double wsum = 0.0, t1[2] = {0.0, 0.0}, t2[2] = {0.0, 0.0};
  for (int sweep = 0; sweep < 2; ++sweep) {
    int32_t current = element;
    for (size_t step = 0; step < around.size(); ++step) {
      const int i = position(current);
      if (i < 0)
        return finish(-1);
      const int32_t other = tri[3 * current + (sweep == 0 ? (i + 2) % 3 : (i + 1) % 3)];
      const int32_t next = across(current, other);
      if (next < 0) {
        truncate();
        c.element = current;
        return finish(2);
      }
      if (m.tri_mat[next] != mat) {
        const double dx = xy[2 * other] - xy[2 * node], dy = xy[2 * other + 1] - xy[2 * node + 1];
        const double len = std::hypot(dx, dy);
        if (!(len > 0.0))
          return finish(-1);
        const double w = 0.5 / len;
        term(current, other, w, dx / len, dy / len, len);
        wsum += w;
        const double len2 = std::hypot(xy[2 * other] - xy[2 * node], xy[2 * other + 1] - xy[2 * node + 1]);
        double *t = sweep == 0 ? t1 : t2;
        t[0] = (xy[2 * other] - xy[2 * node]) / len2;
        t[1] = (xy[2 * other + 1] - xy[2 * node + 1]) / len2;
        break;
      }
      current = next;
    }
  }
  if (!(wsum > 0.0))
    return finish(-1);
  c.wsum = wsum;
  const bool simple = std::hypot(t1[0], t1[1]) < 0.9 || std::hypot(t2[0], t2[1]) < 0.9 ||
                      (-t1[0] * t2[0] - t1[1] * t2[1]) > 0.985;
  if (simple)
    return finish(1);
  // The fallback reads only |B| of the corner's same-label elements and B of the element.
  truncate();
  for (int32_t e : around)
    if (m.tri_mat[e] == mat)
      term(e, -1, 0.0, 0.0, 0.0, 0.0);
  return finish(3);
}

} // namespace

Status BuildPostprocessPlan(const HostModel &m, const fg_postprocess_options &o, std::vector<double> mask,
                            PostprocessPlan *plan)
{
  *plan = PostprocessPlan{};
  const int32_t N = m.nodes(), E = m.triangles();
  if (static_cast<int32_t>(mask.size()) != N ||
      !std::all_of(mask.begin(), mask.end(), [](double v) { return v == 0 || v == 1; }))
    return Status::kInvalidArgument;
  plan->mask = std::move(mask);
  plan->incident.assign(N, {});
  plan->hx.assign(E, 0.0);
  plan->hy.assign(E, 0.0);
  plan->weight.resize(E);
  plan->cx.resize(E);
  plan->cy.resize(E);
  for (int32_t e = 0; e < E; ++e) {
    const int32_t *t = &m.tri[3 * e];
    for (int l = 0; l < 3; ++l)
      plan->incident[t[l]].push_back(e);
    double area, bx[3], by[3];
    if (!ElementTerms(&m.xy[2 * t[0]], &m.xy[2 * t[1]], &m.xy[2 * t[2]], &area, bx, by))
      return Status::kMeshInvalid;
    for (int l = 0; l < 3; ++l) {
      plan->hx[e] += plan->mask[t[l]] * by[l];
      plan->hy[e] -= plan->mask[t[l]] * bx[l];
    }
    plan->weight[e] = area * m.depth_m;
    plan->cx[e] = (m.xy[2 * t[0]] + m.xy[2 * t[1]] + m.xy[2 * t[2]]) / 3.0;
    plan->cy[e] = (m.xy[2 * t[0] + 1] + m.xy[2 * t[1] + 1] + m.xy[2 * t[2] + 1]) / 3.0;
  }
  if (!(o.airgap_radius_m >= 0.0) || !std::isfinite(o.airgap_radius_m) || o.airgap_angle_count < 0 ||
      (o.airgap_angle_count > 0 && !o.airgap_angles_rad))
    return Status::kInvalidArgument;
  // Elements whose bounding box can reach the probe circle, in element order.
  std::vector<int32_t> candidates;
  const double r2 = o.airgap_radius_m * o.airgap_radius_m;
  const double tol = 64.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, r2);
  for (int32_t e = 0; e < E && o.airgap_angle_count > 0; ++e) {
    const int32_t *t = &m.tri[3 * e];
    double lo[2], hi[2];
    for (int d = 0; d < 2; ++d) {
      lo[d] = std::min({m.xy[2 * t[0] + d], m.xy[2 * t[1] + d], m.xy[2 * t[2] + d]});
      hi[d] = std::max({m.xy[2 * t[0] + d], m.xy[2 * t[1] + d], m.xy[2 * t[2] + d]});
    }
    const double nx = lo[0] > 0.0 ? lo[0] : (hi[0] < 0.0 ? hi[0] : 0.0);
    const double ny = lo[1] > 0.0 ? lo[1] : (hi[1] < 0.0 ? hi[1] : 0.0);
    const double fx = std::max(std::abs(lo[0]), std::abs(hi[0]));
    const double fy = std::max(std::abs(lo[1]), std::abs(hi[1]));
    if (r2 + tol >= nx * nx + ny * ny && r2 <= fx * fx + fy * fy + tol)
      candidates.push_back(e);
  }
  const Select sel{o, m};
  for (int32_t k = 0; k < o.airgap_angle_count; ++k) {
    const double angle = o.airgap_angles_rad[k];
    if (!std::isfinite(angle))
      return Status::kInvalidArgument;
    AirgapProbe probe;
    probe.cosine = std::cos(angle);
    probe.sine = std::sin(angle);
    const double x = o.airgap_radius_m * probe.cosine, y = o.airgap_radius_m * probe.sine;
    for (int32_t e : candidates) {
      double cand[3] = {};
      if (Barycentric(m, e, x, y, cand) && cand[0] >= -1e-12 && cand[1] >= -1e-12 && cand[2] >= -1e-12) {
        probe.element = e;
        std::copy(cand, cand + 3, probe.lambda);
        break;
      }
    }
    if (probe.element < 0 || !sel.air(m.tri_mat[probe.element]))
      return Status::kInvalidArgument;
    plan->probes.push_back(probe);
  }
  for (const AirgapProbe &p : plan->probes)
    for (int l = 0; l < 3; ++l)
      BuildCorner(m, p.element, l, plan);
  return Status::kOk;
}

namespace
{

// Probe samples from accessors; false on a smoothing failure.
template <class A, class B1, class B2>
bool Samples(const HostModel &m, const PostprocessPlan &plan, const A &a, const B1 &b1, const B2 &b2,
             double *radial_b)
{
  for (size_t k = 0; k < plan.probes.size(); ++k) {
    const AirgapProbe &p = plan.probes[k];
    double nbx[3] = {}, nby[3] = {};
    if (!NodalB(m, a, b1, b2, plan.incident, p.element, nbx, nby))
      return false;
    double bx = 0.0, by = 0.0;
    for (int l = 0; l < 3; ++l) {
      bx += p.lambda[l] * nbx[l];
      by += p.lambda[l] * nby[l];
    }
    radial_b[k] = bx * p.cosine + by * p.sine;
  }
  return true;
}

} // namespace

Status ComputePostprocess(const HostModel &m, const PostprocessPlan &plan, const double *a, const double *b1,
                          const double *b2, fg_postprocess_result *res, double *radial_b)
{
  res->force_x_n = res->force_y_n = res->torque_nm = 0.0;
  const int32_t E = m.triangles();
  for (int32_t e = 0; e < E; ++e) {
    const double hx = plan.hx[e], hy = plan.hy[e];
    const double bx = b1[e], by = b2[e];
    const double fxd = ((bx * bx - by * by) * hx + 2.0 * bx * by * hy) / (2.0 * kMu0);
    const double fyd = (2.0 * bx * by * hx + (by * by - bx * bx) * hy) / (2.0 * kMu0);
    const double w = plan.weight[e];
    res->force_x_n += w * fxd;
    res->force_y_n += w * fyd;
    res->torque_nm += w * (plan.cx[e] * fyd - plan.cy[e] * fxd);
  }
  auto at = [](const double *v) { return [v](int32_t i) { return v[i]; }; };
  if (!Samples(m, plan, at(a), at(b1), at(b2), radial_b))
    return Status::kMeshInvalid;
  if (!std::isfinite(res->force_x_n) || !std::isfinite(res->force_y_n) || !std::isfinite(res->torque_nm))
    return Status::kNumericalNonfinite;
  return Status::kOk;
}

Status ComputeTangentPostprocess(const HostModel &m, const PostprocessPlan &plan, const double *b1,
                                 const double *b2, const double *da, const double *db1, const double *db2,
                                 fg_postprocess_result *res, double *radial_b)
{
  res->force_x_n = res->force_y_n = res->torque_nm = 0.0;
  const int32_t E = m.triangles();
  for (int32_t e = 0; e < E; ++e) {
    const double hx = plan.hx[e], hy = plan.hy[e];
    const double bx = b1[e], by = b2[e], dbx = db1[e], dby = db2[e];
    const double dnormal = 2.0 * (bx * dbx - by * dby);
    const double dshear = 2.0 * (dbx * by + bx * dby);
    const double dfx = (dnormal * hx + dshear * hy) / (2.0 * kMu0);
    const double dfy = (dshear * hx - dnormal * hy) / (2.0 * kMu0);
    const double w = plan.weight[e];
    res->force_x_n += w * dfx;
    res->force_y_n += w * dfy;
    res->torque_nm += w * (plan.cx[e] * dfy - plan.cy[e] * dfx);
  }
  auto at = [](const double *v) { return [v](int32_t i) { return v[i]; }; };
  if (!Samples(m, plan, at(da), at(db1), at(db2), radial_b))
    return Status::kMeshInvalid;
  if (!std::isfinite(res->force_x_n) || !std::isfinite(res->force_y_n) || !std::isfinite(res->torque_nm))
    return Status::kNumericalNonfinite;
  return Status::kOk;
}

} // namespace fg

using fg::Status;
using fg::ToInt;

extern "C" {

void fg_postprocess_default_options(fg_postprocess_options *o)
{
  if (!o)
    return;
  *o = fg_postprocess_options{};
  o->selected_material_label = 1;
  o->air_material_label = 3;
  o->selected_group_number = -1;
  o->air_group_number = -1;
  o->max_mask_iterations = 256;
  o->mask_relative_tolerance = 1e-12;
}

int fg_postprocess_create(const fg_plan *plan, const fg_postprocess_options *options, const double *mask,
                          fg_postprocess **out)
{
  if (!out)
    return ToInt(Status::kInvalidArgument);
  *out = nullptr;
  if (!plan || !options)
    return ToInt(Status::kInvalidArgument);
  const fg::HostModel &m = plan->plan.model();
  if (m.problem_type != FG_PLANAR)
    return ToInt(Status::kUnsupportedFeature);
  if (!(m.depth_m > 0.0))
    return ToInt(Status::kInvalidArgument);
  try {
    std::vector<double> values;
    if (mask) {
      values.assign(mask, mask + m.nodes());
    } else {
      const Status s = fg::WeightedStressMask(m, *options, &values);
      if (s != Status::kOk)
        return ToInt(s);
    }
    auto *pp = new fg_postprocess;
    pp->model.problem_type = m.problem_type;
    pp->model.xy = m.xy;
    pp->model.tri = m.tri;
    pp->model.tri_mat = m.tri_mat;
    pp->model.depth_m = m.depth_m;
    const Status s = fg::BuildPostprocessPlan(m, *options, std::move(values), &pp->plan);
    if (s != Status::kOk) {
      delete pp;
      return ToInt(s);
    }
    *out = pp;
    return ToInt(Status::kOk);
  } catch (...) {
    return ToInt(Status::kInternalError);
  }
}

void fg_postprocess_destroy(fg_postprocess *pp) { delete pp; }

int32_t fg_postprocess_probe_count(const fg_postprocess *pp)
{
  return pp ? static_cast<int32_t>(pp->plan.probes.size()) : 0;
}

int fg_postprocess_mask(const fg_postprocess *pp, double *mask)
{
  if (!pp || !mask)
    return ToInt(Status::kInvalidArgument);
  std::copy(pp->plan.mask.begin(), pp->plan.mask.end(), mask);
  return ToInt(Status::kOk);
}

int fg_postprocess_compute(const fg_postprocess *pp, int32_t items, const double *a, const double *b1,
                           const double *b2, fg_postprocess_result *results, double *radial)
{
  const size_t P = pp ? pp->plan.probes.size() : 0;
  if (!pp || items < 0 || (items > 0 && (!a || !b1 || !b2 || !results || (P > 0 && !radial))))
    return ToInt(Status::kInvalidArgument);
  const size_t N = pp->model.nodes(), E = pp->model.triangles();
  for (int32_t i = 0; i < items; ++i) {
    fg_postprocess_result &r = results[i];
    r = fg_postprocess_result{};
    r.status = ToInt(fg::ComputePostprocess(pp->model, pp->plan, a + i * N, b1 + i * E, b2 + i * E, &r,
                                            P ? radial + i * P : nullptr));
  }
  return ToInt(Status::kOk);
}

int fg_postprocess_compute_device(fg_postprocess *pp, int32_t items, const double *a, const double *b1,
                                  const double *b2, fg_postprocess_result *results, double *radial,
                                  void *stream_ptr)
{
  const size_t P = pp ? pp->plan.probes.size() : 0;
  if (!pp || items < 0 || (items > 0 && (!a || !b1 || !b2 || !results || (P > 0 && !radial))))
    return ToInt(Status::kInvalidArgument);
  if (items == 0)
    return ToInt(Status::kOk);
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices < 1) {
    cudaGetLastError();
    return ToInt(Status::kGpuUnavailable);
  }
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const fg::PostprocessPlan &pl = pp->plan;
  const int32_t E = pp->model.triangles(), N = pp->model.nodes();
  const int32_t Pn = static_cast<int32_t>(P), T = static_cast<int32_t>(pl.term_elem.size());
  for (const fg::CornerStencil &c : pl.corners)
    if (c.kind < 0) {
      for (int32_t i = 0; i < items; ++i) {
        results[i] = fg_postprocess_result{};
        results[i].status = ToInt(Status::kMeshInvalid);
      }
      return ToInt(Status::kOk);
    }
  Status s = Status::kOk;
  if (pp->geometry.capacity() == 0) {
    std::vector<double> g;
    g.reserve(5 * static_cast<size_t>(E) + 5 * P + 4 * static_cast<size_t>(T));
    for (const std::vector<double> *v : {&pl.hx, &pl.hy, &pl.weight, &pl.cx, &pl.cy})
      g.insert(g.end(), v->begin(), v->end());
    for (const fg::AirgapProbe &p : pl.probes) {
      g.insert(g.end(), p.lambda, p.lambda + 3);
      g.push_back(p.cosine);
      g.push_back(p.sine);
    }
    for (const std::vector<double> *v : {&pl.term_w, &pl.term_tx, &pl.term_ty, &pl.term_len})
      g.insert(g.end(), v->begin(), v->end());
    std::vector<int32_t> ids(pl.term_elem);
    ids.insert(ids.end(), pl.term_node.begin(), pl.term_node.end());
    s = pp->geometry.upload(g.data(), g.size(), stream);
    if (s == Status::kOk)
      s = pp->terms.upload(ids.data(), ids.size(), stream);
    if (s == Status::kOk)
      s = pp->corners.upload(pl.corners.data(), pl.corners.size(), stream);
    // The uploads read pageable host vectors that die here.
    if (s == Status::kOk && cudaStreamSynchronize(stream) != cudaSuccess)
      s = Status::kInternalError;
    if (s != Status::kOk) {
      pp->geometry.reset();
      return ToInt(s);
    }
  }
  const int ctas = fg::PostprocessCtas(E, items);
  const size_t partial_count = static_cast<size_t>(ctas) * items * 3;
  const size_t total = partial_count + P * items;
  if ((s = pp->out.ensure(total)) != Status::kOk || (s = pp->host_out.ensure(total)) != Status::kOk)
    return ToInt(s);
  fg::PostprocessDevice d{};
  const double *g = pp->geometry.get();
  d.hx = g;
  d.hy = g + E;
  d.weight = g + 2 * static_cast<size_t>(E);
  d.cx = g + 3 * static_cast<size_t>(E);
  d.cy = g + 4 * static_cast<size_t>(E);
  d.probe = g + 5 * static_cast<size_t>(E);
  d.term_w = d.probe + 5 * P;
  d.term_tx = d.term_w + T;
  d.term_ty = d.term_tx + T;
  d.term_len = d.term_ty + T;
  d.term_elem = pp->terms.get();
  d.term_node = d.term_elem + T;
  d.corners = pp->corners.get();
  d.E = E;
  d.N = N;
  d.items = items;
  d.ctas = ctas;
  d.probes = Pn;
  d.a = a;
  d.b1 = b1;
  d.b2 = b2;
  d.partials = pp->out.get();
  d.radial = d.partials + partial_count;
  if (fg::LaunchPostprocess(d, stream) != cudaSuccess ||
      cudaMemcpyAsync(pp->host_out.get(), pp->out.get(), total * sizeof(double), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    cudaGetLastError();
    return ToInt(Status::kInternalError);
  }
  const double *h = pp->host_out.get();
  for (int32_t i = 0; i < items; ++i) {
    fg_postprocess_result &r = results[i];
    r = fg_postprocess_result{};
    for (int c = 0; c < ctas; ++c) {
      const double *q = h + (static_cast<size_t>(c) * items + i) * 3;
      r.force_x_n += q[0];
      r.force_y_n += q[1];
      r.torque_nm += q[2];
    }
    if (P)
      std::copy(h + partial_count + P * i, h + partial_count + P * (i + 1), radial + P * i);
    r.status = ToInt(std::isfinite(r.force_x_n) && std::isfinite(r.force_y_n) && std::isfinite(r.torque_nm)
                         ? Status::kOk
                         : Status::kNumericalNonfinite);
  }
  return ToInt(Status::kOk);
}

int fg_postprocess_tangent(const fg_postprocess *pp, int32_t m, const double *b1, const double *b2, const double *da,
                           const double *db1, const double *db2, fg_postprocess_result *results, double *radial)
{
  const size_t P = pp ? pp->plan.probes.size() : 0;
  if (!pp || m < 0 || (m > 0 && (!b1 || !b2 || !da || !db1 || !db2 || !results || (P > 0 && !radial))))
    return ToInt(Status::kInvalidArgument);
  const size_t N = pp->model.nodes(), E = pp->model.triangles();
  for (int32_t i = 0; i < m; ++i) {
    fg_postprocess_result &r = results[i];
    r = fg_postprocess_result{};
    r.status = ToInt(fg::ComputeTangentPostprocess(pp->model, pp->plan, b1, b2, da + i * N, db1 + i * E,
                                                   db2 + i * E, &r, P ? radial + i * P : nullptr));
  }
  return ToInt(Status::kOk);
}

int fg_postprocess_frozen(const fg_plan *plan, const fg_postprocess_options *options, const double *a,
                          const double *b1, const double *b2, fg_postprocess_result *result, double *radial)
{
  if (!result)
    return ToInt(Status::kInvalidArgument);
  *result = fg_postprocess_result{};
  if (!plan || !options || !a || !b1 || !b2 || (options->airgap_angle_count > 0 && !radial))
    return ToInt(Status::kInvalidArgument);
  fg_postprocess *pp = nullptr;
  const int s = fg_postprocess_create(plan, options, nullptr, &pp);
  if (s != 0) {
    result->status = s;
    return ToInt(Status::kOk);
  }
  const int rc = fg_postprocess_compute(pp, 1, a, b1, b2, result, radial);
  fg_postprocess_destroy(pp);
  return rc;
}

} // extern "C"
