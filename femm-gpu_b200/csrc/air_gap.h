// air_gap.h -- FEMM's native air-gap element (AGE): the fixed linear stiffness of an
// untriangulated annular band between a rotor ring and a stator ring of mesh nodes.
#pragma once

#include <cstdint>
#include <vector>

namespace fg
{

// AirGapElement (gpu_solver/src/physics/nonlinear_model.h:63-81).  Point p of the band
// carries node[4 p + l] / weight[4 p + l], l = 0, 1 the inner-ring nodes bracketing it and
// l = 2, 3 the outer-ring ones; a weight is the +1 / -1 sign of the ring copy.
struct AirGap {
  bool antiperiodic = false;
  double cx = 0.0, cy = 0.0, ri = 0.0, ro = 0.0, arc_deg = 0.0;
  double inner_shift = 0.0, outer_shift = 0.0;
  std::vector<int32_t> node;
  std::vector<double> weight;
  int32_t points() const { return static_cast<int32_t>(node.size() / 4); }
  int32_t arcs() const { return points() - 1; }
};

// The band's per-arc constants: K = (ro - ri) / (r_mean dt) (the arc's radial over
// circumferential extent), Ki = 1 / K, and the two ring offsets brought to the form the
// element uses: one side's offset is 0 or 1, the other's is the relative slide in (0, 1]
// (prob1big.cpp's normalisation, physics/nonlinear_topology.cpp:183-194).
struct AirGapTerms {
  double K = 0.0, Ki = 0.0, ci = 0.0, co = 0.0;
};
AirGapTerms AirGapBandTerms(const AirGap &band);

// The 10 x 10 element matrix of one arc in relative-reluctivity units (multiply by 1/mu0),
// over the stencil of AirGapStencil.  Returns false for non-finite or non-positive terms.
//
// Derivation.  The arc is a four-corner element in (theta, r): corners at its two end
// angles on the inner and outer radii.  Each corner value is the cubic Catmull-Rom
// interpolation of four consecutive ring nodes of its side at the fraction t = 1 - c of
// the ring spacing (c = ci or co), the left corner from ring nodes 0..3 of the side's
// five-node stencil and the right corner from nodes 1..4.  With circumferential corner
// differences a = u_ir - u_il, b = u_or - u_ol and radial ones a' = u_ol - u_il,
// b' = u_or - u_ir, the element energy is
//   K  (5 a^2  + 2 a b   + 5 b^2) / 12  +  Ki (5 a'^2 + 2 a' b' + 5 b'^2) / 12,
// i.e. per direction the bilinear quadrilateral's mean-gradient term (a + b)^2 / 4 with
// twice its twist term, (a - b)^2 / 6.  The matrix is T^T Q T with T the 4 x 10
// interpolation and Q the 4 x 4 corner form.  This reproduces FEMM's AGE matrix (its
// expanded polynomials in fkn/prob1big.cpp:158-213) to rounding.
bool AirGapElementMatrix(double K, double Ki, double ci, double co, double m[10][10]);

// The ten (node, weight) pairs of arc k: five consecutive inner-ring nodes, then five
// outer-ring ones (physics/nonlinear_topology.cpp:199-219), with the anti-periodic
// closure's extra sign on the stencil ends that wrap around the band.
void AirGapStencil(const AirGap &band, int32_t k, int32_t node[10], double weight[10]);

// B at the centre of every arc of a band from nodal A [N]: br radial, bt circumferential.
// The arc's corner potentials come from the same Catmull-Rom ring interpolation as the
// stiffness, at t = 1 - (the side's own shift), so the arcs sit on the band's absolute
// angular grid; then Br = (1/r) dA/dtheta and Bt = -dA/dr are the corner differences
// averaged over the arc.  Returns false if a value is not finite.
bool AirGapArcFields(const AirGap &band, const double *a, std::vector<double> *br, std::vector<double> *bt);

// The radial-B Fourier series of a band's arc values, as FEMM's viewer builds it for
// mo_getgapb: the harmonics a periodic (all) or anti-periodic (odd) band carries, in units
// of the band's repeat; value at angle theta = sum_h c_h cos(n_h theta) + s_h sin(n_h theta).
struct AirGapSeries {
  std::vector<int32_t> order;
  std::vector<double> c, s;
  double At(double theta) const;
};
AirGapSeries AirGapRadialSeries(const AirGap &band, const std::vector<double> &br);

// Maxwell-stress force / torque of the band and the series' radial B at the given angles
// (ComputeAirGapElementPostprocess, postprocess/airgap_postprocess.cpp:44-161).  Status as
// the reference: INVALID_ARGUMENT without a band or for a non-finite angle, MESH_INVALID for
// a degenerate band, NUMERICAL_NONFINITE for non-finite fields or totals.
struct AirGapPostResult {
  int32_t status = 0;
  double fx = 0.0, fy = 0.0, torque = 0.0;
  std::vector<double> radial;
};
AirGapPostResult AirGapPostprocess(const std::vector<AirGap> &bands, double depth_m, const double *a,
                                   const std::vector<double> &angles);

// The first-order change of the same quantities along a tangent dA at the base A
// (ComputeAirGapElementTangentPostprocess, airgap_postprocess.cpp:163-285): force and torque
// bilinear in (B, dB), the radial series of dBr.
AirGapPostResult AirGapTangentPostprocess(const std::vector<AirGap> &bands, double depth_m, const double *a,
                                          const double *da, const std::vector<double> &angles);

} // namespace fg
