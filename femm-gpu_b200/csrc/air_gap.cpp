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

bool AirGapArcFields(const AirGap &band, const double *a, std::vector<double> *br, std::vector<double> *bt)
{
  const int32_t arcs = band.arcs();
  const double dt = (kPi / 180.0) * band.arc_deg / static_cast<double>(arcs);
  const double radius = 0.5 * (band.ri + band.ro), dr = band.ro - band.ri;
  double wi[4], wo[4];
  CatmullRom(1.0 - band.inner_shift, wi);
  CatmullRom(1.0 - band.outer_shift, wo);
  br->assign(arcs, 0.0);
  bt->assign(arcs, 0.0);
  for (int32_t k = 0; k < arcs; ++k) {
    int32_t node[10];
    double weight[10], v[10];
    AirGapStencil(band, k, node, weight);
    for (int i = 0; i < 10; ++i)
      v[i] = a[node[i]] * weight[i];
    double il = 0.0, ir = 0.0, ol = 0.0, orr = 0.0;
    for (int l = 0; l < 4; ++l) {
      il += wi[l] * v[l];
      ir += wi[l] * v[l + 1];
      ol += wo[l] * v[5 + l];
      orr += wo[l] * v[6 + l];
    }
    (*br)[k] = ((ir - il) + (orr - ol)) / (2.0 * dt * radius);
    (*bt)[k] = ((il + ir) - (ol + orr)) / (2.0 * dr);
    if (!std::isfinite((*br)[k]) || !std::isfinite((*bt)[k]))
      return false;
  }
  return true;
}

double AirGapSeries::At(double theta) const
{
  double v = 0.0;
  for (size_t h = 0; h < order.size(); ++h) {
    const double phase = static_cast<double>(order[h]) * theta;
    v += c[h] * std::cos(phase) + s[h] * std::sin(phase);
  }
  return v;
}

AirGapSeries AirGapRadialSeries(const AirGap &band, const std::vector<double> &br)
{
  // A periodic band of arc span S repeats every S: harmonics 0, 1, 2, ... in units of
  // 360/S, up to Nyquist.  An anti-periodic one changes sign every S: odd multiples of
  // 180/S only.  DC and the Nyquist term of an even periodic count have weight 1/arcs,
  // the others 2/arcs (a real DFT at the arc centres).
  const int32_t arcs = band.arcs();
  const double dt = (kPi / 180.0) * band.arc_deg / static_cast<double>(arcs);
  const size_t count = band.antiperiodic ? static_cast<size_t>((arcs + 1) / 2) : static_cast<size_t>(arcs / 2 + 1);
  const int32_t base = static_cast<int32_t>(std::lround((band.antiperiodic ? 180.0 : 360.0) / band.arc_deg));
  AirGapSeries f;
  f.order.resize(count);
  f.c.assign(count, 0.0);
  f.s.assign(count, 0.0);
  for (size_t h = 0; h < count; ++h) {
    const int32_t n = band.antiperiodic ? base * static_cast<int32_t>(2 * h + 1) : base * static_cast<int32_t>(h);
    f.order[h] = n;
    for (int32_t k = 0; k < arcs; ++k) {
      const double phase = (static_cast<double>(k) + 0.5) * dt * static_cast<double>(n);
      f.c[h] += br[k] * std::cos(phase);
      f.s[h] += br[k] * std::sin(phase);
    }
    const bool single = n == 0 || (!band.antiperiodic && h + 1 == count && arcs % 2 == 0);
    const double norm = single ? static_cast<double>(arcs) : static_cast<double>(arcs) / 2.0;
    f.c[h] /= norm;
    f.s[h] /= norm;
  }
  return f;
}

namespace
{

bool BandGeometry(const AirGap &band, double *dt, double *radius)
{
  *dt = (kPi / 180.0) * band.arc_deg / static_cast<double>(band.arcs());
  *radius = 0.5 * (band.ri + band.ro);
  return *dt > 0.0 && *radius > 0.0 && band.ro - band.ri > 0.0;
}

} // namespace

AirGapPostResult AirGapPostprocess(const std::vector<AirGap> &bands, double depth_m, const double *a,
                                   const std::vector<double> &angles)
{
  AirGapPostResult r;
  if (bands.empty() || !a) {
    r.status = static_cast<int32_t>(Status::kInvalidArgument);
    return r;
  }
  AirGapSeries first;
  for (size_t b = 0; b < bands.size(); ++b) {
    const AirGap &band = bands[b];
    double dt, radius;
    if (band.arcs() < 2 || !BandGeometry(band, &dt, &radius)) {
      r.status = static_cast<int32_t>(Status::kMeshInvalid);
      return r;
    }
    std::vector<double> br, bt;
    if (!AirGapArcFields(band, a, &br, &bt)) {
      r.status = static_cast<int32_t>(Status::kNumericalNonfinite);
      return r;
    }
    // Maxwell stress on the band's mid circle: normal (Br^2 - Bt^2) / 2mu0 and shear
    // Br Bt / mu0 per unit area, resolved at each arc centre.
    const double scale = depth_m * radius * dt / (2.0 * kMu0);
    for (int32_t k = 0; k < band.arcs(); ++k) {
      const double theta = (static_cast<double>(k) + 0.5) * dt;
      const double normal = br[k] * br[k] - bt[k] * bt[k], shear = 2.0 * br[k] * bt[k];
      r.fx += scale * (normal * std::cos(theta) - shear * std::sin(theta));
      r.fy += scale * (normal * std::sin(theta) + shear * std::cos(theta));
      r.torque += depth_m * radius * radius * dt * br[k] * bt[k] / kMu0;
    }
    if (b == 0)
      first = AirGapRadialSeries(band, br);
  }
  for (const double angle : angles) {
    if (!std::isfinite(angle)) {
      r.status = static_cast<int32_t>(Status::kInvalidArgument);
      return r;
    }
    r.radial.push_back(first.At(angle));
  }
  if (!std::isfinite(r.fx) || !std::isfinite(r.fy) || !std::isfinite(r.torque))
    r.status = static_cast<int32_t>(Status::kNumericalNonfinite);
  return r;
}

AirGapPostResult AirGapTangentPostprocess(const std::vector<AirGap> &bands, double depth_m, const double *a,
                                          const double *da, const std::vector<double> &angles)
{
  AirGapPostResult r;
  if (bands.empty() || !a || !da) {
    r.status = static_cast<int32_t>(Status::kInvalidArgument);
    return r;
  }
  AirGapSeries first;
  for (size_t b = 0; b < bands.size(); ++b) {
    const AirGap &band = bands[b];
    double dt, radius;
    if (band.arcs() < 2 || !BandGeometry(band, &dt, &radius)) {
      r.status = static_cast<int32_t>(Status::kMeshInvalid);
      return r;
    }
    std::vector<double> br, bt, dbr, dbt;
    AirGapArcFields(band, a, &br, &bt);
    AirGapArcFields(band, da, &dbr, &dbt);
    const double scale = depth_m * radius * dt / (2.0 * kMu0);
    for (int32_t k = 0; k < band.arcs(); ++k) {
      const double theta = (static_cast<double>(k) + 0.5) * dt;
      const double dnormal = 2.0 * (br[k] * dbr[k] - bt[k] * dbt[k]);
      const double dshear = 2.0 * (dbr[k] * bt[k] + br[k] * dbt[k]);
      r.fx += scale * (dnormal * std::cos(theta) - dshear * std::sin(theta));
      r.fy += scale * (dnormal * std::sin(theta) + dshear * std::cos(theta));
      r.torque += depth_m * radius * radius * dt * (dbr[k] * bt[k] + br[k] * dbt[k]) / kMu0;
    }
    if (b == 0)
      first = AirGapRadialSeries(band, dbr);
  }
  for (const double angle : angles)
    r.radial.push_back(first.At(angle));
  r.status = std::isfinite(r.fx) && std::isfinite(r.fy) && std::isfinite(r.torque)
                 ? 0
                 : static_cast<int32_t>(Status::kNumericalNonfinite);
  return r;
}

} // namespace fg
