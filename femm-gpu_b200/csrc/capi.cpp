// capi.cpp -- the extern "C" boundary (include/femm_gpu.h).
#include "femm_gpu.h"
#include "solver.h"
#include "warm.h"
#include "multi.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <vector>

using fg::Status;
using fg::ToInt;

namespace
{

Status ToHostModel(const fg_model *m, fg::HostModel *out)
{
  if (!m || m->node_count <= 0 || m->triangle_count <= 0 || m->material_count <= 0 || !m->node_xy ||
      !m->triangle_nodes || !m->triangle_material || !m->materials || m->curve_count < 0 ||
      (m->curve_count > 0 && !m->curves) || m->dirichlet_count < 0 ||
      (m->dirichlet_count > 0 && (!m->dirichlet_nodes || !m->dirichlet_values)) ||
      m->constraint_count < 0 ||
      (m->constraint_count > 0 && (!m->constraint_nodes || !m->constraint_signs)))
    return Status::kInvalidArgument;
  fg::HostModel h;
  h.problem_type = m->problem_type;
  if (h.problem_type != FG_PLANAR && h.problem_type != FG_AXISYMMETRIC)
    return Status::kInvalidArgument;
  h.xy.assign(m->node_xy, m->node_xy + 2 * static_cast<size_t>(m->node_count));
  h.tri.assign(m->triangle_nodes, m->triangle_nodes + 3 * static_cast<size_t>(m->triangle_count));
  h.tri_mat.assign(m->triangle_material, m->triangle_material + m->triangle_count);
  for (int i = 0; i < m->material_count; ++i) {
    const fg_material &s = m->materials[i];
    fg::Material mt;
    mt.nu0 = s.reluctivity_zero_m_per_h;
    mt.alpha = s.alpha_per_t2;
    mt.j_per_a = s.source_j_per_a;
    mt.hc = s.h_c_a_per_m;
    mt.deg = s.magnetization_deg;
    mt.curve = s.bh_curve_index;
    mt.circuit = s.circuit_index;
    mt.group = s.group_number;
    h.materials.push_back(mt);
  }
  for (int c = 0; c < m->curve_count; ++c) {
    const fg_bh_curve &src = m->curves[c];
    if (src.count < 2 || src.count > 4096 || !src.b_t || !src.h_a_per_m)
      return Status::kInvalidMaterial;
    fg::BhCurve curve;
    curve.b.assign(src.b_t, src.b_t + src.count);
    curve.h.assign(src.h_a_per_m, src.h_a_per_m + src.count);
    if (!fg::BuildBhSpline(&curve))
      return Status::kInvalidMaterial;
    h.curves.push_back(std::move(curve));
  }
  h.dir_nodes.assign(m->dirichlet_nodes, m->dirichlet_nodes + m->dirichlet_count);
  h.dir_values.assign(m->dirichlet_values, m->dirichlet_values + m->dirichlet_count);
  for (int i = 0; i < m->constraint_count; ++i) {
    h.con_a.push_back(m->constraint_nodes[2 * i]);
    h.con_b.push_back(m->constraint_nodes[2 * i + 1]);
    h.con_sign.push_back(m->constraint_signs[i]);
  }
  h.circuit_count = m->circuit_count;
  h.depth_m = m->depth_m;
  if (m->air_gap_count < 0 || (m->air_gap_count > 0 && !m->air_gap_elements))
    return Status::kInvalidArgument;
  for (int i = 0; i < m->air_gap_count; ++i) {
    const fg_air_gap_element &src = m->air_gap_elements[i];
    if (src.point_count < 0 || (src.point_count > 0 && (!src.nodes || !src.weights)))
      return Status::kInvalidArgument;
    fg::AirGap g;
    g.antiperiodic = src.antiperiodic != 0;
    g.cx = src.center_x_m;
    g.cy = src.center_y_m;
    g.ri = src.inner_radius_m;
    g.ro = src.outer_radius_m;
    g.arc_deg = src.arc_length_deg;
    g.inner_shift = src.inner_shift;
    g.outer_shift = src.outer_shift;
    g.node.assign(src.nodes, src.nodes + 4 * static_cast<size_t>(src.point_count));
    g.weight.assign(src.weights, src.weights + 4 * static_cast<size_t>(src.point_count));
    h.ages.push_back(std::move(g));
  }
  *out = std::move(h);
  return Status::kOk;
}

} // namespace

extern "C" {

void fg_production_options(fg_solve_options *o)
{
  if (!o)
    return;
  o->relative_tolerance = 1e-8;
  o->max_newton_iterations = 128;
  o->max_linear_iterations = 16384;
  o->linear_relative_tolerance = 1e-10;
  o->recover_nonconvergence = 1;
  o->adaptive_linear_tolerance = 1;
}

const char *fg_status_name(int status)
{
  if (status < 0 || status > 15)
    return "INTERNAL_ERROR";
  return fg::StatusName(static_cast<Status>(status));
}

int fg_abi_version(void) { return FG_ABI_VERSION; }

int64_t fg_set_wait_limit_ns(int64_t ns) { return fg::SetPcgWaitLimitNs(ns); }

int fg_plan_create(const fg_model *model, const fg_plan_options *options, fg_plan **plan)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  *plan = nullptr;
  fg::HostModel h;
  Status s = ToHostModel(model, &h);
  if (s != Status::kOk)
    return ToInt(s);
  fg_plan_options opts{};
  if (options)
    opts = *options;
  fg_plan *p = new (std::nothrow) fg_plan;
  if (!p)
    return ToInt(Status::kInternalError);
  s = p->plan.Create(std::move(h), opts);
  if (s != Status::kOk) {
    delete p;
    return ToInt(s);
  }
  *plan = p;
  return 0;
}

void fg_plan_destroy(fg_plan *plan) { delete plan; }

int fg_plan_sizes_get(const fg_plan *plan, fg_plan_sizes *sizes)
{
  if (!plan || !sizes)
    return ToInt(Status::kInvalidArgument);
  const fg::HostPlan &h = plan->plan.host();
  sizes->node_count = h.N;
  sizes->triangle_count = h.E;
  sizes->rows = h.n;
  sizes->nnz = h.nnz;
  sizes->circuit_count = h.C;
  sizes->problem_type = h.problem_type;
  sizes->device_bytes = static_cast<int64_t>(plan->plan.DeviceBytes());
  sizes->matrix_contributors = static_cast<int64_t>(h.contrib.size());
  sizes->rhs_contributors = static_cast<int64_t>(h.rhs_contrib.size());
  return 0;
}

int fg_plan_contributors(const fg_plan *plan, int32_t *slot_offsets, int32_t *slot_entries,
                         int32_t *row_offsets, int32_t *row_entries, double *pm_rhs,
                         double *circuit_rhs)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  const fg::HostPlan &h = plan->plan.host();
  if (slot_offsets)
    std::copy(h.contrib_off.begin(), h.contrib_off.end(), slot_offsets);
  if (slot_entries)
    for (size_t k = 0; k < h.contrib.size(); ++k) {
      slot_entries[3 * k] = h.contrib[k] >> 4;
      slot_entries[3 * k + 1] = (h.contrib[k] >> 1) & 7;
      slot_entries[3 * k + 2] = (h.contrib[k] & 1) ? -1 : 1;
    }
  if (row_offsets)
    std::copy(h.rhs_off.begin(), h.rhs_off.end(), row_offsets);
  if (row_entries)
    for (size_t k = 0; k < h.rhs_contrib.size(); ++k) {
      row_entries[3 * k] = h.rhs_contrib[k] >> 3;
      row_entries[3 * k + 1] = (h.rhs_contrib[k] >> 1) & 3;
      row_entries[3 * k + 2] = (h.rhs_contrib[k] & 1) ? -1 : 1;
    }
  if (pm_rhs)
    std::copy(h.pm_rhs.begin(), h.pm_rhs.end(), pm_rhs);
  if (circuit_rhs)
    std::copy(h.circuit_rhs.begin(), h.circuit_rhs.end(), circuit_rhs);
  return 0;
}

int fg_plan_air_gap(const fg_plan *plan, double *values, double *rhs)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  const fg::HostPlan &h = plan->plan.host();
  if (values) {
    if (h.age_val.empty())
      std::fill(values, values + h.nnz, 0.0);
    else
      std::copy(h.age_val.begin(), h.age_val.end(), values);
  }
  if (rhs) {
    if (h.age_rhs.empty())
      std::fill(rhs, rhs + h.n, 0.0);
    else
      std::copy(h.age_rhs.begin(), h.age_rhs.end(), rhs);
  }
  return 0;
}

int fg_plan_symbolic(const fg_plan *plan, int32_t *row_offsets, int32_t *columns,
                     int32_t *node_to_free, int8_t *node_sign, double *boundary_values)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  const fg::HostPlan &h = plan->plan.host();
  if (row_offsets)
    std::copy(h.row_offsets.begin(), h.row_offsets.end(), row_offsets);
  if (columns)
    std::copy(h.columns.begin(), h.columns.end(), columns);
  if (node_to_free)
    std::copy(h.dofs.node_to_free.begin(), h.dofs.node_to_free.end(), node_to_free);
  if (node_sign)
    std::copy(h.dofs.node_sign.begin(), h.dofs.node_sign.end(), node_sign);
  if (boundary_values)
    std::copy(h.dofs.boundary.begin(), h.dofs.boundary.end(), boundary_values);
  return 0;
}

int fg_assemble(fg_plan *plan, int32_t items, const double *states, const double *currents,
                const int32_t *use_newton, double *values, double *diagonal, double *rhs)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  return ToInt(plan->plan.Assemble(items, states, currents, use_newton, values, diagonal, rhs));
}

int fg_pcg_solve(fg_plan *plan, int32_t items, const double *values, int32_t values_per_item,
                 const double *rhs, double relative_tolerance, int32_t max_iterations, double *x,
                 fg_linear_info *info)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  return ToInt(plan->plan.PcgSolve(items, values, values_per_item, rhs, relative_tolerance,
                                   max_iterations, x, info));
}

int fg_plan_attach_device(fg_plan *plan)
{
  if (!plan)
    return ToInt(Status::kInvalidArgument);
  try {
    return ToInt(plan->plan.AttachDevice());
  } catch (...) {
    return ToInt(Status::kInternalError);
  }
}

int fg_solve_tangent(fg_plan *plan, const double *base_a, const double *base_currents, int32_t directions,
                     const double *direction_currents, const fg_solve_options *options, double *da,
                     double *db1, double *db2, double *dflux, fg_linear_info *info)
{
  if (!plan || !options)
    return ToInt(Status::kInvalidArgument);
  try {
    return ToInt(plan->plan.SolveTangent(base_a, base_currents, directions, direction_currents, *options, da, db1,
                                         db2, dflux, info));
  } catch (...) {
    return ToInt(Status::kInternalError);
  }
}

int fg_solve_batch(fg_plan *plan, int32_t items, const double *currents, const double *hc_scale,
                   const double *warm_a, const fg_solve_options *options, double *a_out,
                   double *b1_out, double *b2_out, double *flux_out, fg_item_info *info)
{
  if (!plan || !options)
    return ToInt(Status::kInvalidArgument);
  return ToInt(plan->plan.SolveHost(items, currents, hc_scale, warm_a, *options, a_out, b1_out,
                                    b2_out, flux_out, info));
}

int fg_multi_create(fg_plan *const *plans, int32_t count, fg_multi **multi)
{
  if (!plans || count <= 0 || !multi)
    return ToInt(Status::kInvalidArgument);
  *multi = nullptr;
  std::vector<fg::Plan *> list;
  for (int32_t i = 0; i < count; ++i) {
    if (!plans[i])
      return ToInt(Status::kInvalidArgument);
    list.push_back(&plans[i]->plan);
  }
  auto *m = new (std::nothrow) fg_multi;
  if (!m)
    return ToInt(Status::kInternalError);
  const Status s = m->solver.Create(std::move(list));
  if (s != Status::kOk) {
    delete m;
    return ToInt(s);
  }
  *multi = m;
  return 0;
}

void fg_multi_destroy(fg_multi *multi) { delete multi; }

int fg_multi_solve(fg_multi *multi, const double *const *currents, const fg_solve_options *options,
                   double *const *a_out, double *const *b1_out, double *const *b2_out,
                   double *const *flux_out, fg_item_info *info)
{
  if (!multi || !options || !info)
    return ToInt(Status::kInvalidArgument);
  return ToInt(multi->solver.Solve(currents, *options, a_out, b1_out, b2_out, flux_out, info));
}

int fg_multi_last_timing(const fg_multi *multi, fg_multi_timing *timing)
{
  if (!multi || !timing)
    return ToInt(Status::kInvalidArgument);
  *timing = multi->solver.timing();
  return 0;
}

int fg_mlp_create(int32_t inputs, int32_t hidden, int32_t outputs, uint64_t seed, fg_mlp **mlp)
{
  if (!mlp)
    return ToInt(Status::kInvalidArgument);
  *mlp = nullptr;
  auto *m = new (std::nothrow) fg_mlp;
  if (!m)
    return ToInt(Status::kInternalError);
  const Status s = m->mlp.Create(inputs, hidden, outputs, seed);
  if (s != Status::kOk) {
    delete m;
    return ToInt(s);
  }
  *mlp = m;
  return 0;
}

void fg_mlp_destroy(fg_mlp *mlp) { delete mlp; }

int64_t fg_mlp_parameter_count(const fg_mlp *mlp) { return mlp ? mlp->mlp.ParameterCount() : 0; }

int fg_mlp_get_parameters(const fg_mlp *mlp, float *parameters)
{
  if (!mlp || !parameters)
    return ToInt(Status::kInvalidArgument);
  return ToInt(mlp->mlp.GetParameters(parameters));
}

int fg_mlp_set_parameters(fg_mlp *mlp, const float *parameters)
{
  if (!mlp || !parameters)
    return ToInt(Status::kInvalidArgument);
  return ToInt(mlp->mlp.SetParameters(parameters));
}

int fg_mlp_forward(fg_mlp *mlp, int32_t batch, const float *x, float *y)
{
  if (!mlp)
    return ToInt(Status::kInvalidArgument);
  return ToInt(mlp->mlp.Predict(batch, x, y));
}

int fg_mlp_loss_gradient(fg_mlp *mlp, int32_t batch, const float *x, const float *t, float *loss,
                         float *gradient)
{
  if (!mlp)
    return ToInt(Status::kInvalidArgument);
  return ToInt(mlp->mlp.LossGradient(batch, x, t, loss, gradient));
}

int fg_mlp_train(fg_mlp *mlp, int32_t samples, const float *x, const float *t, int32_t epochs,
                 int32_t batch, float learning_rate, uint64_t seed, float *final_loss)
{
  if (!mlp)
    return ToInt(Status::kInvalidArgument);
  return ToInt(mlp->mlp.Train(samples, x, t, epochs, batch, learning_rate, seed, final_loss));
}

int fg_warm_create(const fg_plan *plan, int32_t rank, const double *mean, const double *basis,
                   fg_mlp *mlp, const float *feature_shift, const float *feature_scale,
                   const double *coeff_shift, const double *coeff_scale, fg_warm **warm)
{
  if (!plan || !warm)
    return ToInt(Status::kInvalidArgument);
  *warm = nullptr;
  auto *w = new (std::nothrow) fg_warm;
  if (!w)
    return ToInt(Status::kInternalError);
  const Status s = w->warm.Create(plan->plan.host().N, rank, mean, basis, mlp ? &mlp->mlp : nullptr,
                                  feature_shift, feature_scale, coeff_shift, coeff_scale);
  if (s != Status::kOk) {
    delete w;
    return ToInt(s);
  }
  *warm = w;
  return 0;
}

void fg_warm_destroy(fg_warm *warm) { delete warm; }

int fg_warm_project(fg_warm *warm, int32_t k, const double *a, double *coeffs)
{
  if (!warm)
    return ToInt(Status::kInvalidArgument);
  return ToInt(warm->warm.Project(k, a, coeffs));
}

int fg_warm_project_device(fg_warm *warm, int32_t k, const double *a, double *coeffs, void *stream)
{
  if (!warm || !a || !coeffs)
    return ToInt(Status::kInvalidArgument);
  return ToInt(warm->warm.ProjectDevice(k, a, coeffs, static_cast<cudaStream_t>(stream)));
}

int fg_warm_predict(fg_warm *warm, int32_t k, const float *features, double *a)
{
  if (!warm)
    return ToInt(Status::kInvalidArgument);
  return ToInt(warm->warm.Predict(k, features, a));
}

int fg_solve_batch_learned(fg_plan *plan, fg_warm *warm, int32_t items, const double *currents,
                           const double *hc_scale, const float *features,
                           const fg_solve_options *options, double *a_out, double *b1_out,
                           double *b2_out, double *flux_out, fg_item_info *info)
{
  if (!plan || !warm || !options || !features || !info || items <= 0 || warm->warm.inputs() == 0 ||
      warm->warm.N() != plan->plan.host().N)
    return ToInt(Status::kInvalidArgument);
  const fg::HostPlan &h = plan->plan.host();
  const size_t N = h.N, E = h.E, C = h.C;
  const int I = warm->warm.inputs();
  Status s;
  if ((s = warm->features.upload(features, static_cast<size_t>(items) * I)) != Status::kOk)
    return ToInt(s);
  // Warm starts are predicted chunk by chunk (kMaxItems items) into one reused buffer.
  for (int first = 0; first < items; first += fg::kMaxItems) {
    const int k = std::min(fg::kMaxItems, items - first);
    if ((s = warm->starts.ensure(static_cast<size_t>(k) * N)) != Status::kOk ||
        (s = warm->warm.PredictDevice(k, warm->features.get() + static_cast<size_t>(first) * I,
                                      warm->starts.get(), nullptr)) != Status::kOk)
      return ToInt(s);
    s = plan->plan.SolveHost(k, currents ? currents + first * C : nullptr,
                             hc_scale ? hc_scale + first : nullptr, nullptr, *options,
                             a_out ? a_out + first * N : nullptr, b1_out ? b1_out + first * E : nullptr,
                             b2_out ? b2_out + first * E : nullptr,
                             flux_out ? flux_out + first * C : nullptr, info + first,
                             warm->starts.get(), true);
    if (s != Status::kOk)
      return ToInt(s);
  }
  return 0;
}

int fg_solve_batch_device(fg_plan *plan, int32_t items, const double *currents,
                          const double *hc_scale, const double *warm_a,
                          const fg_solve_options *options, double *a_out, double *b1_out,
                          double *b2_out, double *flux_out, fg_item_info *info, void *stream)
{
  if (!plan || !options)
    return ToInt(Status::kInvalidArgument);
  fg::SolveRequest r;
  r.items = items;
  r.currents = currents;
  r.hc_scale = hc_scale;
  r.warm = warm_a;
  r.options = *options;
  r.a_out = a_out;
  r.b1_out = b1_out;
  r.b2_out = b2_out;
  r.flux_out = flux_out;
  r.info = info;
  r.stream = static_cast<cudaStream_t>(stream);
  return ToInt(plan->plan.SolveDevice(r));
}

int fg_plan_last_timing(const fg_plan *plan, fg_timing *timing)
{
  if (!plan || !timing)
    return ToInt(Status::kInvalidArgument);
  *timing = plan->plan.timing();
  return 0;
}

int fg_plan_pcg_shapes(const fg_plan *plan, int32_t capacity, fg_pcg_shape *shapes)
{
  if (!plan || capacity < 0 || (capacity > 0 && !shapes))
    return 0;
  const auto &all = plan->plan.pcg_shapes();
  int32_t n = 0;
  for (const auto &entry : all) {
    if (n < capacity)
      shapes[n] = entry.second;
    ++n;
  }
  return n;
}

int fg_bh_build(int32_t count, double *b, double *h, double *slope, double *cold_secant,
                int32_t *smoothing_passes)
{
  if (count < 2 || !b || !h || !slope)
    return 0;
  fg::BhCurve c;
  c.b.assign(b, b + count);
  c.h.assign(h, h + count);
  if (!fg::BuildBhSpline(&c))
    return 0;
  std::copy(c.b.begin(), c.b.end(), b);
  std::copy(c.h.begin(), c.h.end(), h);
  std::copy(c.slope.begin(), c.slope.end(), slope);
  if (cold_secant)
    *cold_secant = c.cold_secant;
  if (smoothing_passes)
    *smoothing_passes = c.smoothing_passes;
  return 1;
}

void fg_bh_eval(int32_t count, const double *b, const double *h, const double *slope,
                double field_b, double *out)
{
  fg::BhCurve c;
  c.b.assign(b, b + count);
  c.h.assign(h, h + count);
  c.slope.assign(slope, slope + count);
  fg::EvaluateBh(c, field_b, out);
}

int fg_air_gap_postprocess(const fg_plan *plan, int32_t items, const double *a, int32_t angle_count,
                           const double *angles_rad, fg_postprocess_result *results,
                           double *airgap_radial_b_t)
{
  if (!plan || items < 0 || !results || (items > 0 && !a) || angle_count < 0 ||
      (angle_count > 0 && (!angles_rad || !airgap_radial_b_t)))
    return ToInt(Status::kInvalidArgument);
  const fg::HostModel &m = plan->plan.model();
  const std::vector<double> angles(angles_rad, angles_rad + angle_count);
  const size_t N = static_cast<size_t>(m.nodes());
  for (int32_t i = 0; i < items; ++i) {
    const fg::AirGapPostResult r = fg::AirGapPostprocess(m.ages, m.depth_m, a + i * N, angles);
    results[i] = fg_postprocess_result{r.status, 0, r.fx, r.fy, r.torque};
    for (int32_t j = 0; j < angle_count; ++j)
      airgap_radial_b_t[static_cast<size_t>(i) * angle_count + j] =
          j < static_cast<int32_t>(r.radial.size()) ? r.radial[j] : 0.0;
  }
  return 0;
}

int fg_air_gap_tangent(const fg_plan *plan, int32_t directions, const double *base_a, const double *da,
                       int32_t angle_count, const double *angles_rad, fg_postprocess_result *results,
                       double *airgap_radial_b_t)
{
  if (!plan || directions < 0 || !results || !base_a || (directions > 0 && !da) || angle_count < 0 ||
      (angle_count > 0 && (!angles_rad || !airgap_radial_b_t)))
    return ToInt(Status::kInvalidArgument);
  const fg::HostModel &m = plan->plan.model();
  const std::vector<double> angles(angles_rad, angles_rad + angle_count);
  const size_t N = static_cast<size_t>(m.nodes());
  for (int32_t i = 0; i < directions; ++i) {
    const fg::AirGapPostResult r = fg::AirGapTangentPostprocess(m.ages, m.depth_m, base_a, da + i * N, angles);
    results[i] = fg_postprocess_result{r.status, 0, r.fx, r.fy, r.torque};
    for (int32_t j = 0; j < angle_count; ++j)
      airgap_radial_b_t[static_cast<size_t>(i) * angle_count + j] =
          j < static_cast<int32_t>(r.radial.size()) ? r.radial[j] : 0.0;
  }
  return 0;
}

} // extern "C"
