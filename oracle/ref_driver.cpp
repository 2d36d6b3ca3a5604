// ref_driver.cpp -- C entry points over the REFERENCE's own host sources.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// FEMM-GPU's host translation units where they lie in the reference checkout
// (gpu_solver/src/physics/{nonlinear_model,linear_model,nonlinear_topology}.cpp,
// core/types.cpp, io/{strict_json,mesh_artifact}.cpp, postprocess/{field_postprocess.cpp,
// weighted_stress.cu} and the FEMM fixture reader tests/native/reference.cpp) into
// oracle/_ref/libfemm_ref.so.  weighted_stress.cu is compiled as host C++ against
// shim_cuda/solvers/csr_solver.cuh, a CPU stand-in for its one GPU linear solve.
// Tests use it to pin the C restatement (femm_oracle.c) and the product's host
// preparation to the reference bit for bit; nothing in the product loads it.
#include "physics/nonlinear_model.h"
#include "physics/nonlinear_topology.h"
#include "io/mesh_artifact.h"
#include "io/sample_request.h"
#include "io/strict_json.h"
#include "postprocess/postprocess.h"
#include "signed_node_constraints.h"
#include "../tests/native/reference.h"

#include "femm_oracle.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace gpu_femm;

// FEMM's native air-gap element matrix (native_airgap_matrix.cpp, its body cut from
// fkn/prob1big.cpp by the Makefile as the reference's own build does).
bool BuildNativeFemmAirGapMatrix(double K, double Ki, double ci, double co, double matrix[10][10]);

namespace
{

bool ToModel(const or_model *m, NonlinearModel *out)
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
  for (int i = 0; i < m->age_count; ++i) {
    const or_air_gap &src = m->ages[i];
    AirGapElement age;
    age.antiperiodic = src.antiperiodic != 0;
    age.center_x_m = src.center_x_m;
    age.center_y_m = src.center_y_m;
    age.inner_radius_m = src.inner_radius_m;
    age.outer_radius_m = src.outer_radius_m;
    age.arc_length_deg = src.arc_length_deg;
    age.inner_shift = src.inner_shift;
    age.outer_shift = src.outer_shift;
    for (int p = 0; p < src.point_count; ++p) {
      AirGapQuadPoint point;
      for (int l = 0; l < 4; ++l) {
        point.node[l] = src.nodes[4 * p + l];
        point.weight[l] = src.weights[4 * p + l];
      }
      age.quad_points.push_back(point);
    }
    model.air_gap_elements.push_back(std::move(age));
  }
  *out = std::move(model);
  return true;
}

} // namespace

// The one oracle-model -> NonlinearModel conversion, shared with ref_cpu_baseline.cpp.
bool RefModelFromOracle(const or_model *m, NonlinearModel *out) { return ToModel(m, out); }

struct ref_system {
  Assembly assembly;
};

struct ref_prepared {
  PreparedNonlinearAssembly prepared;
};

struct ref_artifact {
  GpuFemmMeshArtifact artifact;
  std::string error;
  // FEMM fixtures read by ReadNonlinearFemmReference: FEMM's nodal A and flux linkage.
  std::vector<double> expected_a;
  double flux_linkage_wb = 0.0;
};

extern "C" {

int ref_bh_build(int32_t n, double *b, double *h, double *slope, double *cold, int32_t *passes)
{
  NonlinearBhCurve curve;
  curve.b_t.assign(b, b + n);
  curve.h_a_per_m.assign(h, h + n);
  if (!BuildNonlinearBhSpline(&curve))
    return 0;
  std::memcpy(b, curve.b_t.data(), sizeof(double) * n);
  std::memcpy(h, curve.h_a_per_m.data(), sizeof(double) * n);
  std::memcpy(slope, curve.slope.data(), sizeof(double) * n);
  *cold = curve.cold_secant_reluctivity_m_per_h;
  *passes = curve.smoothing_passes;
  return 1;
}

void ref_bh_eval(int32_t n, const double *b, const double *h, const double *slope, double field,
                 double *out)
{
  NonlinearBhCurve curve;
  curve.b_t.assign(b, b + n);
  curve.h_a_per_m.assign(h, h + n);
  curve.slope.assign(slope, slope + n);
  const NonlinearBhEvaluation e = EvaluateNonlinearBh(curve, field);
  out[0] = e.h_a_per_m;
  out[1] = e.dh_db;
  out[2] = e.reluctivity_m_per_h;
  out[3] = e.dv_db2;
}

int ref_validate(const or_model *m)
{
  NonlinearModel model;
  if (!ToModel(m, &model))
    return static_cast<int>(Status::kInvalidMaterial);
  return static_cast<int>(ValidateNonlinearModel(model));
}

int ref_assemble(const or_model *m, const double *a_old, const double *currents, int use_newton,
                 ref_system **out)
{
  *out = nullptr;
  NonlinearModel model;
  if (!ToModel(m, &model))
    return static_cast<int>(Status::kInvalidMaterial);
  auto system = std::make_unique<ref_system>();
  const Status status = AssembleNonlinearNewton(
      model, std::vector<double>(a_old, a_old + m->node_count),
      std::vector<double>(currents, currents + m->circuit_count), use_newton != 0,
      &system->assembly);
  if (status != Status::kOk)
    return static_cast<int>(status);
  *out = system.release();
  return 0;
}

int32_t ref_system_rows(const ref_system *s) { return (int32_t)s->assembly.free_nodes.size(); }
int32_t ref_system_nnz(const ref_system *s) { return (int32_t)s->assembly.values.size(); }

void ref_system_copy(const ref_system *s, int32_t *row_offsets, int32_t *columns, double *values,
                     double *diagonal, double *rhs, int32_t *node_to_free, int8_t *node_sign,
                     double *boundary)
{
  const Assembly &a = s->assembly;
  if (row_offsets)
    std::memcpy(row_offsets, a.row_offsets.data(), sizeof(int32_t) * a.row_offsets.size());
  if (columns)
    std::memcpy(columns, a.column_indices.data(), sizeof(int32_t) * a.column_indices.size());
  if (values)
    std::memcpy(values, a.values.data(), sizeof(double) * a.values.size());
  if (diagonal)
    std::memcpy(diagonal, a.diagonal.data(), sizeof(double) * a.diagonal.size());
  if (rhs)
    for (size_t r = 0; r < a.rhs_per_amp.size(); ++r)
      rhs[r] = a.rhs_per_amp[r] + a.rhs_offset[r];
  if (node_to_free)
    std::memcpy(node_to_free, a.node_to_free.data(), sizeof(int32_t) * a.node_to_free.size());
  if (node_sign)
    std::memcpy(node_sign, a.node_sign.data(), a.node_sign.size());
  if (boundary)
    std::memcpy(boundary, a.boundary_values.data(), sizeof(double) * a.boundary_values.size());
}

void ref_system_free(ref_system *s) { delete s; }

// Device-assembly plan topology (nonlinear_topology.cpp:12-248): symbolic CSR,
// per-slot contributor lists, per-row RHS contributor lists and pre-summed loads.
int ref_prepare(const or_model *m, ref_prepared **out)
{
  *out = nullptr;
  NonlinearModel model;
  if (!ToModel(m, &model))
    return static_cast<int>(Status::kInvalidMaterial);
  auto prepared = std::make_unique<ref_prepared>();
  const Status status = PrepareNonlinearAssembly(model, &prepared->prepared);
  if (status != Status::kOk)
    return static_cast<int>(status);
  *out = prepared.release();
  return 0;
}

int32_t ref_prepared_rows(const ref_prepared *p) { return (int32_t)p->prepared.symbolic.free_nodes.size(); }
int32_t ref_prepared_nnz(const ref_prepared *p) { return (int32_t)p->prepared.symbolic.column_indices.size(); }
int32_t ref_prepared_matrix_entries(const ref_prepared *p) { return (int32_t)p->prepared.matrix_entries.size(); }
int32_t ref_prepared_rhs_entries(const ref_prepared *p) { return (int32_t)p->prepared.rhs_entries.size(); }

// matrix_entries as (triangle, local_row, local_column, sign) quadruples; rhs as triples.
void ref_prepared_copy(const ref_prepared *p, int32_t *row_offsets, int32_t *columns,
                       int32_t *free_nodes, int32_t *matrix_offsets, int32_t *matrix_entries,
                       int32_t *rhs_offsets, int32_t *rhs_entries, double *pm_rhs,
                       double *circuit_rhs, int32_t *diagonal_slots)
{
  const PreparedNonlinearAssembly &q = p->prepared;
  std::memcpy(row_offsets, q.symbolic.row_offsets.data(), sizeof(int32_t) * q.symbolic.row_offsets.size());
  std::memcpy(columns, q.symbolic.column_indices.data(), sizeof(int32_t) * q.symbolic.column_indices.size());
  std::memcpy(free_nodes, q.symbolic.free_nodes.data(), sizeof(int32_t) * q.symbolic.free_nodes.size());
  std::memcpy(matrix_offsets, q.matrix_offsets.data(), sizeof(int32_t) * q.matrix_offsets.size());
  for (size_t k = 0; k < q.matrix_entries.size(); ++k) {
    matrix_entries[4 * k] = q.matrix_entries[k].triangle;
    matrix_entries[4 * k + 1] = q.matrix_entries[k].local_row;
    matrix_entries[4 * k + 2] = q.matrix_entries[k].local_column;
    matrix_entries[4 * k + 3] = q.matrix_entries[k].sign;
  }
  std::memcpy(rhs_offsets, q.rhs_offsets.data(), sizeof(int32_t) * q.rhs_offsets.size());
  for (size_t k = 0; k < q.rhs_entries.size(); ++k) {
    rhs_entries[3 * k] = q.rhs_entries[k].triangle;
    rhs_entries[3 * k + 1] = q.rhs_entries[k].local_row;
    rhs_entries[3 * k + 2] = q.rhs_entries[k].sign;
  }
  std::memcpy(pm_rhs, q.pm_rhs.data(), sizeof(double) * q.pm_rhs.size());
  std::memcpy(circuit_rhs, q.circuit_rhs.data(), sizeof(double) * q.circuit_rhs.size());
  std::memcpy(diagonal_slots, q.diagonal_slots.data(), sizeof(int32_t) * q.diagonal_slots.size());
}

// PreparedNonlinearAssembly::age_values [nnz] / age_rhs [rows] (nonlinear_topology.cpp:180-262).
void ref_prepared_age(const ref_prepared *p, double *age_values, double *age_rhs)
{
  std::memcpy(age_values, p->prepared.age_values.data(), sizeof(double) * p->prepared.age_values.size());
  std::memcpy(age_rhs, p->prepared.age_rhs.data(), sizeof(double) * p->prepared.age_rhs.size());
}

void ref_prepared_free(ref_prepared *p) { delete p; }

int ref_signed_dofs(int32_t node_count, int32_t con_count, const int32_t *ca, const int32_t *cb,
                    const int8_t *cs, int32_t dir_count, const int32_t *dn, const double *dv,
                    int32_t *node_root, int8_t *node_sign, int32_t *root_to_free,
                    int32_t *free_count)
{
  std::vector<SignedNodeConstraint> constraints;
  for (int i = 0; i < con_count; ++i) {
    SignedNodeConstraint c;
    c.node_a = ca[i];
    c.node_b = cb[i];
    c.sign = cs[i];
    constraints.push_back(c);
  }
  SignedDofMap map;
  const SignedDofStatus status = BuildSignedDofMap(
      node_count, constraints, std::vector<int32_t>(dn, dn + dir_count),
      std::vector<double>(dv, dv + dir_count), &map);
  if (status != SignedDofStatus::kOk)
    return static_cast<int>(status);
  for (int i = 0; i < node_count; ++i) {
    node_root[i] = map.node_root[i];
    node_sign[i] = map.node_sign[i];
    root_to_free[i] = map.root_to_free[i];
  }
  *free_count = (int32_t)map.free_roots.size();
  return 0;
}

// Strict artifact parse (mesh_artifact.cpp:14-715) of a JSON text.
int ref_parse_artifact(const char *text, size_t length, ref_artifact **out)
{
  auto artifact = std::make_unique<ref_artifact>();
  const bool ok =
      ParseGpuFemmMeshArtifactJson(std::string(text, length), &artifact->artifact, &artifact->error);
  *out = artifact.release();
  return ok ? 0 : 1;
}

const char *ref_artifact_error(const ref_artifact *a) { return a->error.c_str(); }

// sizes[8] = nodes, triangles, materials, curves, dirichlet, constraints, circuits, curve points
void ref_artifact_sizes(const ref_artifact *a, int32_t *sizes, double *depth_m, int32_t *problem_type)
{
  const NonlinearModel &m = a->artifact.model;
  sizes[0] = (int32_t)m.nodes.size();
  sizes[1] = (int32_t)m.triangles.size();
  sizes[2] = (int32_t)m.materials.size();
  sizes[3] = (int32_t)m.bh_curves.size();
  sizes[4] = (int32_t)m.dirichlet_nodes.size();
  sizes[5] = (int32_t)m.node_constraints.size();
  sizes[6] = m.circuit_count;
  int32_t points = 0;
  for (const auto &c : m.bh_curves)
    points += (int32_t)c.b_t.size();
  sizes[7] = points;
  *depth_m = m.depth_m;
  *problem_type = m.problem_type == MagneticProblemType::kAxisymmetric ? 1 : 0;
}

// materials: [M x 5] doubles (nu0, alpha, J/A, Hc, deg) and [M x 3] ints (curve, circuit, group).
void ref_artifact_copy(const ref_artifact *a, double *xy, int32_t *tri, int32_t *tri_mat,
                       double *mat_d, int32_t *mat_i, double *curve_b, double *curve_h,
                       double *curve_slope, int32_t *dir_nodes, int32_t *con, double *currents)
{
  const NonlinearModel &m = a->artifact.model;
  for (size_t i = 0; i < m.nodes.size(); ++i) {
    xy[2 * i] = m.nodes[i].x_m;
    xy[2 * i + 1] = m.nodes[i].y_m;
  }
  for (size_t e = 0; e < m.triangles.size(); ++e) {
    for (int l = 0; l < 3; ++l)
      tri[3 * e + l] = m.triangles[e].node[l];
    tri_mat[e] = m.triangles[e].material;
  }
  for (size_t i = 0; i < m.materials.size(); ++i) {
    const NonlinearMaterial &mt = m.materials[i];
    mat_d[5 * i] = mt.reluctivity_zero_m_per_h;
    mat_d[5 * i + 1] = mt.alpha_per_t2;
    mat_d[5 * i + 2] = mt.source_j_per_a;
    mat_d[5 * i + 3] = mt.h_c_a_per_m;
    mat_d[5 * i + 4] = mt.magnetization_deg;
    mat_i[3 * i] = mt.bh_curve_index;
    mat_i[3 * i + 1] = mt.circuit_index;
    mat_i[3 * i + 2] = mt.group_number;
  }
  size_t k = 0;
  for (const auto &c : m.bh_curves)
    for (size_t p = 0; p < c.b_t.size(); ++p, ++k) {
      curve_b[k] = c.b_t[p];
      curve_h[k] = c.h_a_per_m[p];
      curve_slope[k] = c.slope[p];
    }
  for (size_t i = 0; i < m.dirichlet_nodes.size(); ++i)
    dir_nodes[i] = m.dirichlet_nodes[i];
  for (size_t i = 0; i < m.node_constraints.size(); ++i) {
    con[3 * i] = m.node_constraints[i].node_a;
    con[3 * i + 1] = m.node_constraints[i].node_b;
    con[3 * i + 2] = m.node_constraints[i].sign;
  }
  for (size_t i = 0; i < a->artifact.circuit_currents_a.size(); ++i)
    currents[i] = a->artifact.circuit_currents_a[i];
}

void ref_artifact_free(ref_artifact *a) { delete a; }

void ref_sha256(const char *bytes, size_t length, char *hex65)
{
  const std::string hex = Sha256Hex(std::string(bytes, length));
  std::memcpy(hex65, hex.c_str(), 65);
}

int ref_canonical_sha256(const char *json, size_t length, char *hex65)
{
  StrictJson root;
  std::string error;
  const std::string text(json, length);
  StrictJsonParser parser(text);
  if (!parser.Parse(&root, &error))
    return 1;
  const std::string hex = CanonicalJsonSha256(root);
  std::memcpy(hex65, hex.c_str(), 65);
  return 0;
}

// ReadSingleSampleRequest (io/sample_request.cpp:98-135).  Returns 0 and fills the fields
// (strings into 4096-byte buffers, angles into [64]) or 1 and the error text in `error`.
int ref_read_single_sample_request(const char *path, char *stem, char *curve_directory, char *sha,
                                   double *current_a, int32_t *selected_label, double *radius_mm,
                                   int32_t *angle_count, double *angles_deg, char *error)
{
  SingleSampleRequest r;
  std::string e;
  if (!ReadSingleSampleRequest(path, &r, &e)) {
    std::snprintf(error, 4096, "%s", e.c_str());
    return 1;
  }
  std::snprintf(stem, 4096, "%s", r.stem.c_str());
  std::snprintf(curve_directory, 4096, "%s", r.curve_directory.c_str());
  std::snprintf(sha, 4096, "%s", r.source_motor_fem_sha256.c_str());
  *current_a = r.current_a;
  *selected_label = r.selected_material_label;
  *radius_mm = r.airgap_radius_mm;
  *angle_count = static_cast<int32_t>(r.airgap_angles_deg.size());
  for (size_t i = 0; i < r.airgap_angles_deg.size() && i < 64; ++i)
    angles_deg[i] = r.airgap_angles_deg[i];
  return 0;
}

// A model handle for ref_postprocess from an oracle model; groups [materials] or NULL.
int ref_model_handle(const or_model *m, const int32_t *groups, ref_artifact **out)
{
  auto h = std::make_unique<ref_artifact>();
  if (!ToModel(m, &h->artifact.model)) {
    *out = h.release();
    return 1;
  }
  if (groups)
    for (size_t i = 0; i < h->artifact.model.materials.size(); ++i)
      h->artifact.model.materials[i].group_number = groups[i];
  *out = h.release();
  return 0;
}

// NonlinearModel::symmetry_apex_nodes (physics/nonlinear_model.h:96) of a model handle: the
// Dirichlet nodes the weighted-stress mask does not hold at 0 (weighted_stress.cu:80-84).
void ref_model_set_apex(ref_artifact *h, int32_t count, const int32_t *nodes)
{
  h->artifact.model.symmetry_apex_nodes.assign(nodes, nodes + count);
}

// ReadNonlinearFemmReference (tests/native/reference.cpp:229-379): a FEMM .ans solution
// with the fixture's hard-wired materials, as a model handle for ref_artifact_sizes / copy.
int ref_read_femm_nonlinear(const char *stem, const char *curve_directory, ref_artifact **out)
{
  auto h = std::make_unique<ref_artifact>();
  NonlinearFemmReference reference;
  if (!ReadNonlinearFemmReference(stem, curve_directory, &reference, &h->error)) {
    *out = h.release();
    return 1;
  }
  h->artifact.model = std::move(reference.model);
  h->artifact.circuit_currents_a = {reference.current_a};
  h->expected_a = std::move(reference.expected_a);
  h->flux_linkage_wb = reference.flux_linkage_wb;
  *out = h.release();
  return 0;
}

void ref_femm_expected(const ref_artifact *h, double *a, double *flux_linkage_wb)
{
  std::copy(h->expected_a.begin(), h->expected_a.end(), a);
  *flux_linkage_wb = h->flux_linkage_wb;
}

// ComputeFrozenPostprocess (field_postprocess.cpp:341-403) on a model handle and a given
// solution.  mask [N] (0 / 1) selects BuildFrozenPostprocessPlanWithMask, NULL the full
// BuildFrozenPostprocessPlan (mask through weighted_stress.cu); mask_out [N] may be NULL.
// out3 = Fx, Fy, torque; radial [angles].  Returns the result status.
int ref_postprocess(const ref_artifact *h, const double *a, const double *b1, const double *b2,
                    const int32_t *labels /* selected, air, selected group, air group */,
                    double radius_m, int32_t angle_count, const double *angles_rad,
                    int32_t max_mask_iterations, double mask_tolerance, const double *mask,
                    double *out3, double *radial, double *mask_out)
{
  const NonlinearModel &m = h->artifact.model;
  FrozenPostprocessOptions o;
  o.selected_material_label = labels[0];
  o.air_material_label = labels[1];
  o.selected_group_number = labels[2];
  o.air_group_number = labels[3];
  o.airgap_radius_m = radius_m;
  o.airgap_angles_rad.assign(angles_rad, angles_rad + angle_count);
  o.max_mask_iterations = max_mask_iterations;
  o.mask_relative_tolerance = mask_tolerance;
  NonlinearSolveResult solution;
  solution.a_wb_per_m.assign(a, a + m.nodes.size());
  solution.bx_t.assign(b1, b1 + m.triangles.size());
  solution.by_t.assign(b2, b2 + m.triangles.size());
  FrozenPostprocessPlan plan;
  const Status ps = mask ? BuildFrozenPostprocessPlanWithMask(
                               m, o, std::vector<double>(mask, mask + m.nodes.size()), &plan)
                         : BuildFrozenPostprocessPlan(m, o, &plan);
  if (ps != Status::kOk)
    return static_cast<int>(ps);
  if (mask_out)
    std::copy(plan.mask.begin(), plan.mask.end(), mask_out);
  const FrozenPostprocessResult r = ComputeFrozenPostprocess(m, solution, o, &plan);
  out3[0] = r.force_x_n;
  out3[1] = r.force_y_n;
  out3[2] = r.torque_nm;
  for (size_t i = 0; i < r.airgap_samples.size(); ++i)
    radial[i] = r.airgap_samples[i].radial_b_t;
  return static_cast<int>(r.status);
}

// ComputeFrozenTangentPostprocess (field_postprocess.cpp:405-520) with the reusable plan
// built from `mask`: out3 = dFx, dFy, dtorque per amp; radial [angles].  Returns the status.
int ref_tangent_postprocess(const ref_artifact *h, const double *a, const double *b1, const double *b2,
                            const double *da, const double *db1, const double *db2, const int32_t *labels,
                            double radius_m, int32_t angle_count, const double *angles_rad, const double *mask,
                            double *out3, double *radial)
{
  const NonlinearModel &m = h->artifact.model;
  FrozenPostprocessOptions o;
  o.selected_material_label = labels[0];
  o.air_material_label = labels[1];
  o.selected_group_number = labels[2];
  o.air_group_number = labels[3];
  o.airgap_radius_m = radius_m;
  o.airgap_angles_rad.assign(angles_rad, angles_rad + angle_count);
  const std::vector<double> mk(mask, mask + m.nodes.size());
  FrozenPostprocessPlan plan;
  const Status ps = BuildFrozenPostprocessPlanWithMask(m, o, mk, &plan);
  if (ps != Status::kOk)
    return static_cast<int>(ps);
  NonlinearSolveResult base, derivative;
  base.a_wb_per_m.assign(a, a + m.nodes.size());
  base.bx_t.assign(b1, b1 + m.triangles.size());
  base.by_t.assign(b2, b2 + m.triangles.size());
  derivative.a_wb_per_m.assign(da, da + m.nodes.size());
  derivative.bx_t.assign(db1, db1 + m.triangles.size());
  derivative.by_t.assign(db2, db2 + m.triangles.size());
  const TangentPostprocessResult r = ComputeFrozenTangentPostprocess(m, base, derivative, o, mk, &plan);
  out3[0] = r.force_x_n_per_a;
  out3[1] = r.force_y_n_per_a;
  out3[2] = r.torque_nm_per_a;
  for (size_t i = 0; i < r.airgap_radial_flux_density_t_per_a.size(); ++i)
    radial[i] = r.airgap_radial_flux_density_t_per_a[i];
  return static_cast<int>(r.status);
}

// ReadMotorSampleRequestJson (io/sample_request.cpp:212-391) and ReadMotorBatchRequestJson
// (app/batch_prepare.cpp:73-129) are not compiled here (the batch reader sits in a CUDA
// translation unit's neighbourhood); the sample reader is: 0 accepted, 1 refused (error).
int ref_read_motor_sample_request(const char *text, size_t length, char *error)
{
  MotorSampleRequest r;
  std::string e;
  const bool ok = ReadMotorSampleRequestJson(std::string(text, length), &r, &e);
  std::snprintf(error, 4096, "%s", e.c_str());
  return ok ? 0 : 1;
}

} // extern "C"

// BuildNativeFemmAirGapMatrix (native_airgap_matrix.cpp:5-22) as a flat [10][10].
extern "C" int ref_age_matrix(double K, double Ki, double ci, double co, double *out)
{
  double m[10][10];
  if (!BuildNativeFemmAirGapMatrix(K, Ki, ci, co, m))
    return 1;
  std::memcpy(out, m, sizeof(m));
  return 0;
}

int RefCpuNewtonModel(const NonlinearModel &model, int32_t k, const double *currents, const or_options *o,
                      int32_t threads, double *a_out, double *flux_out, int32_t *status,
                      int32_t *newton_iterations, int32_t *pcg_calls, double *max_true_residual);

extern "C" {

// ApplySlidingBandAngle (io/sample_request.cpp:448-491) on a handle: a new handle whose
// model is posed at angle_deg.  A handle built from an oracle model with air-gap elements
// counts as a zero-degree sliding-band artifact.
int ref_sliding_band_pose(const ref_artifact *h, double angle_deg, ref_artifact **out)
{
  auto posed = std::make_unique<ref_artifact>();
  posed->artifact = h->artifact;
  GpuFemmMeshArtifact source = h->artifact;
  if (!source.model.air_gap_elements.empty())
    source.has_sliding_band = true;
  const bool ok = ApplySlidingBandAngle(angle_deg, source, &posed->artifact.model);
  *out = posed.release();
  return ok ? 0 : 1;
}

int32_t ref_age_count(const ref_artifact *h) { return (int32_t)h->artifact.model.air_gap_elements.size(); }

int32_t ref_age_points(const ref_artifact *h, int32_t b)
{
  return (int32_t)h->artifact.model.air_gap_elements[b].quad_points.size();
}

// meta: antiperiodic, center x, center y, ri, ro, arc degrees, inner shift, outer shift.
void ref_age_copy(const ref_artifact *h, int32_t b, double *meta, int32_t *nodes, double *weights)
{
  const AirGapElement &g = h->artifact.model.air_gap_elements[b];
  const double m[8] = {g.antiperiodic ? 1.0 : 0.0, g.center_x_m, g.center_y_m, g.inner_radius_m,
                       g.outer_radius_m, g.arc_length_deg, g.inner_shift, g.outer_shift};
  std::memcpy(meta, m, sizeof(m));
  for (size_t p = 0; p < g.quad_points.size(); ++p)
    for (int l = 0; l < 4; ++l) {
      nodes[4 * p + l] = g.quad_points[p].node[l];
      weights[4 * p + l] = g.quad_points[p].weight[l];
    }
}

// ComputeAirGapElementPostprocess (postprocess/airgap_postprocess.cpp:44-161): out3 = Fx, Fy,
// torque; radial [angle_count].
int ref_age_postprocess(const ref_artifact *h, const double *a, int32_t angle_count, const double *angles_rad,
                        double *out3, double *radial)
{
  NonlinearSolveResult solution;
  solution.a_wb_per_m.assign(a, a + h->artifact.model.nodes.size());
  FrozenPostprocessOptions o;
  o.airgap_angles_rad.assign(angles_rad, angles_rad + angle_count);
  const FrozenPostprocessResult r = ComputeAirGapElementPostprocess(h->artifact.model, solution, o);
  out3[0] = r.force_x_n;
  out3[1] = r.force_y_n;
  out3[2] = r.torque_nm;
  for (size_t i = 0; i < r.airgap_samples.size(); ++i)
    radial[i] = r.airgap_samples[i].radial_b_t;
  return static_cast<int>(r.status);
}

// ComputeAirGapElementTangentPostprocess (airgap_postprocess.cpp:163-285) with the base model
// as the tangent model.
int ref_age_tangent_postprocess(const ref_artifact *h, const double *a, const double *da, int32_t angle_count,
                                const double *angles_rad, double *out3, double *radial)
{
  NonlinearSolveResult base, derivative;
  const size_t N = h->artifact.model.nodes.size();
  base.a_wb_per_m.assign(a, a + N);
  derivative.a_wb_per_m.assign(da, da + N);
  FrozenPostprocessOptions o;
  o.airgap_angles_rad.assign(angles_rad, angles_rad + angle_count);
  const TangentPostprocessResult r =
      ComputeAirGapElementTangentPostprocess(h->artifact.model, h->artifact.model, base, derivative, o);
  out3[0] = r.force_x_n_per_a;
  out3[1] = r.force_y_n_per_a;
  out3[2] = r.torque_nm_per_a;
  for (size_t i = 0; i < r.airgap_radial_flux_density_t_per_a.size(); ++i)
    radial[i] = r.airgap_radial_flux_density_t_per_a[i];
  return static_cast<int>(r.status);
}

// The reference CPU Newton path (ref_cpu_baseline.cpp) on a handle's model.
int ref_artifact_cpu_solve(const ref_artifact *h, int32_t k, const double *currents, const or_options *o,
                           int32_t threads, double *a_out, double *flux_out, int32_t *status,
                           int32_t *newton_iterations)
{
  std::vector<int32_t> calls(k);
  std::vector<double> worst(k);
  return RefCpuNewtonModel(h->artifact.model, k, currents, o, threads, a_out, flux_out, status,
                           newton_iterations, calls.data(), worst.data());
}

} // extern "C"

