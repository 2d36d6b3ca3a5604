// model.h -- host-side model, B-H spline, validation, signed DOF folding and the
// device assembly plan topology.
#pragma once

#include "air_gap.h"
#include "common.h"

#include <cstdint>
#include <string>
#include <vector>

namespace fg
{

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kTwoPi = 6.283185307179586476925286766559005768;
constexpr double kMu0 = 4.0e-7 * kPi;

struct Material {
  double nu0 = 0.0, alpha = 0.0, j_per_a = 0.0, hc = 0.0, deg = 0.0;
  int32_t curve = -1, circuit = -1, group = -1;
};

struct BhCurve {
  std::vector<double> b, h, slope;
  double cold_secant = 0.0;
  int32_t smoothing_passes = 0;
};

struct HostModel {
  int32_t problem_type = 0; // 0 planar, 1 axisymmetric
  std::vector<double> xy;   // [2N]
  std::vector<int32_t> tri; // [3E]
  std::vector<int32_t> tri_mat;
  std::vector<Material> materials;
  std::vector<BhCurve> curves; // splines built
  std::vector<int32_t> dir_nodes;
  std::vector<double> dir_values;
  std::vector<int32_t> con_a, con_b;
  std::vector<int8_t> con_sign;
  int32_t circuit_count = 1;
  double depth_m = 0.0;
  std::vector<AirGap> ages; // native air-gap elements (planar only)

  int32_t nodes() const { return static_cast<int32_t>(xy.size() / 2); }
  int32_t triangles() const { return static_cast<int32_t>(tri_mat.size()); }
};

// FEMM DC natural-cubic B-H spline with 3-point smoothing until monotone
// (gpu_solver/src/physics/nonlinear_model.cpp:13-113).  Returns false if invalid.
bool BuildBhSpline(BhCurve *curve);
// H, dH/dB, nu, dnu/d(B^2) (nonlinear_model.cpp:115-148).
void EvaluateBh(const BhCurve &curve, double field_b, double out[4]);

// P1 element terms (nonlinear_model.cpp:207-221): area and curl basis.
bool ElementTerms(const double *p0, const double *p1, const double *p2, double *area,
                  double bx[3], double by[3]);

// ValidateNonlinearModel (nonlinear_model.cpp:223-319).
Status ValidateModel(const HostModel &model);

// Signed DOF map (signed_node_constraints.h:33-106).
struct SignedDofs {
  std::vector<int32_t> node_root, node_to_free, free_roots;
  std::vector<int8_t> node_sign;
  std::vector<double> boundary; // expanded fixed values per node
};
// 0 ok, 1 invalid constraint, 2 contradictory cycle, 3 invalid fixed value.
int BuildSignedDofs(const HostModel &model, SignedDofs *dofs);

// Host topology of the device assembly (the role of nonlinear_topology.cpp:12-248,
// laid out for the SELL-32 kernels).
struct HostPlan {
  int32_t N = 0, E = 0, n = 0, C = 0, n_pad = 0, slices = 0;
  int64_t nnz = 0, positions = 0;
  int32_t problem_type = 0;
  SignedDofs dofs;
  // Symbolic CSR, columns ascending per row (std::map order of the reference).
  std::vector<int32_t> row_offsets, columns, diag_slot;
  // SELL-32: slice_off[s] = first position of slice s; position = slice_off + w*32 + r%32.
  std::vector<int32_t> slice_off, row_len, sell_col;
  // Matrix contributors per CSR slot in element order: (element << 4) | (pair << 1) | negative.
  std::vector<int32_t> contrib_off, contrib;
  // RHS contributors per free row: (element << 3) | (local << 1) | negative.
  std::vector<int32_t> rhs_off, rhs_contrib;
  std::vector<double> pm_rhs;      // [n]
  std::vector<double> circuit_rhs; // [C * n]
  // Air-gap elements: their fixed stiffness per CSR slot and the load their fixed nodes put
  // on free rows, each summed in band / arc / i / j order (nonlinear_topology.cpp:180-232);
  // empty without air-gap elements.
  std::vector<double> age_val;     // [nnz]
  std::vector<double> age_rhs;     // [n]
  // Element data: node ids, material, planar area and curl basis.
  std::vector<int32_t> elem_nodes; // [3E]
  std::vector<int32_t> elem_mat;   // [E]
  std::vector<double> elem_geo;    // planar: [7][E] = area, bx0..2, by0..2; axisymmetric: [6][E] = r0..2, z0..2
  // Materials (device copy) and curves.
  std::vector<double> mat_nu0, mat_alpha, mat_cold, mat_jpa;
  std::vector<int32_t> mat_curve_off, mat_curve_cnt, mat_circuit;
  std::vector<double> curve_b, curve_h, curve_slope;
  // Circuit element lists for flux recovery: elements sorted by circuit.
  std::vector<int32_t> circuit_elem_off, circuit_elems;
  bool has_nonlinear = false;
};

Status BuildHostPlan(const HostModel &model, HostPlan *plan);

// Symmetric local-pair index of (i, j) in a 3x3 element matrix: 00,01,02,11,12,22.
inline int PairIndex(int i, int j)
{
  static const int table[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  return table[i][j];
}

} // namespace fg
