// air_gap.cpp -- FEMM's native air-gap element, derived as a four-corner element over
// Catmull-Rom ring interpolation (the derivation is in air_gap.h).
#include "air_gap.h"

#include "model.h"

#include <cmath>

namespace fg
{

AirGapTerms AirGapBandTerms(const AirGap &band)
{
  AirGapTerms t;
  const double dt = (kPi / 180.0) * band.arc_deg / static_cast<double>(band.arcs());
  t.K = 2.0 * (band.ro - band.ri) / (dt * (band.ro + band.ri));
  t.Ki = 1.0 / t.K;
  // Measure the slide from the side that lies ahead: that side's corners sit on its ring
  // nodes (offset 0 or 1), the other's between two of them.
  if (band.inner_shift > band.outer_shift) {
    t.ci = band.inner_shift - band.outer_shift;
    t.co = 0.0;
  } else {
    t.ci = 1.0 - band.outer_shift + band.inner_shift;
    t.co = 1.0;
  }
  return t;
}

namespace
{

// Catmull-Rom weights of ring nodes -1, 0, 1, 2 at fraction t of the 0-1 spacing.
void CatmullRom(double t, double w[4])
{
  const double t2 = t * t, t3 = t2 * t;
  w[0] = 0.5 * (-t3 + 2.0 * t2 - t);
  w[1] = 0.5 * (3.0 * t3 - 5.0 * t2 + 2.0);
  w[2] = 0.5 * (-3.0 * t3 + 4.0 * t2 + t);
  w[3] = 0.5 * (t3 - t2);
}

} // namespace

bool AirGapElementMatrix(double K, double Ki, double ci, double co, double m[10][10])
{
  if (!(K > 0.0) || !(Ki > 0.0) || !std::isfinite(K) || !std::isfinite(Ki) || !std::isfinite(ci) ||
      !std::isfinite(co))
    return false;
  // T: corner rows il, ir, ol, or over the ten stencil nodes.
  double T[4][10] = {};
  double wi[4], wo[4];
  CatmullRom(1.0 - ci, wi);
  CatmullRom(1.0 - co, wo);
  for (int l = 0; l < 4; ++l) {
    T[0][l] = wi[l];
    T[1][l + 1] = wi[l];
    T[2][5 + l] = wo[l];
    T[3][6 + l] = wo[l];
  }
  // Q: the corner form K (5a^2 + 2ab + 5b^2)/12 + Ki (5a'^2 + 2a'b' + 5b'^2)/12.
  const double d = 5.0 * (K + Ki) / 12.0, along = (Ki - 5.0 * K) / 12.0, across = (K - 5.0 * Ki) / 12.0,
               diagonal = -(K + Ki) / 12.0;
  const double Q[4][4] = {{d, along, across, diagonal},
                          {along, d, diagonal, across},
                          {across, diagonal, d, along},
                          {diagonal, across, along, d}};
  double QT[4][10];
  for (int a = 0; a < 4; ++a)
    for (int j = 0; j < 10; ++j) {
      double s = 0.0;
      for (int b = 0; b < 4; ++b)
        s += Q[a][b] * T[b][j];
      QT[a][j] = s;
    }
  for (int i = 0; i < 10; ++i)
    for (int j = i; j < 10; ++j) {
      double s = 0.0;
      for (int a = 0; a < 4; ++a)
        s += T[a][i] * QT[a][j];
      m[i][j] = s;
      m[j][i] = s;
    }
  return true;
}

void AirGapStencil(const AirGap &band, int32_t k, int32_t node[10], double weight[10])
{
  const int32_t arcs = band.arcs();
  const int32_t prev = k == 0 ? arcs - 1 : k - 1, next = k + 1, next2 = k + 2 > arcs ? 1 : k + 2;
  // (point, pair) of each stencil entry: inner ring from n0 / n1, outer from n2 / n3.
  const int32_t pt[10] = {prev, k, k, next, next2, prev, k, k, next, next2};
  const int32_t pair[10] = {0, 0, 1, 1, 1, 2, 2, 3, 3, 3};
  for (int i = 0; i < 10; ++i) {
    node[i] = band.node[4 * pt[i] + pair[i]];
    weight[i] = band.weight[4 * pt[i] + pair[i]];
  }
  // The stencil's outer ends reach one ring node past the band's closure: across an
  // anti-periodic closure that node's copy carries the opposite sign.
  if (band.antiperiodic && k == 0) {
    weight[0] = -weight[0];
    weight[5] = -weight[5];
  }
  if (band.antiperiodic && k + 1 == arcs) {
    weight[4] = -weight[4];
    weight[9] = -weight[9];
  }
}

} // namespace fg
