// femm_ans.cpp -- gpu_femm_single_sample_v1 requests and FEMM .ans nonlinear fixtures.
#include "femm_ans.h"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace fgio
{
namespace
{

constexpr double kMu0 = 4.0e-7 * 3.141592653589793238462643383279502884;

// Position of the value after the first "key" and its colon, whitespace skipped.
bool ValueStart(const std::string &json, const std::string &key, size_t *pos)
{
  const std::string quoted = "\"" + key + "\"";
  const size_t at = json.find(quoted);
  if (at == std::string::npos)
    return false;
  const size_t colon = json.find(':', at + quoted.size());
  if (colon == std::string::npos)
    return false;
  *pos = colon + 1;
  while (*pos < json.size() && std::isspace(static_cast<unsigned char>(json[*pos])))
    ++*pos;
  return *pos < json.size();
}

bool LaxString(const std::string &json, const std::string &key, std::string *value)
{
  size_t pos = 0;
  if (!ValueStart(json, key, &pos) || json[pos] != '"')
    return false;
  const size_t end = json.find('"', pos + 1);
  if (end == std::string::npos)
    return false;
  *value = json.substr(pos + 1, end - pos - 1);
  return value->find('\\') == std::string::npos;
}

// strtod prefix of json[pos..]; 0 characters consumed = no number.
bool Number(const std::string &json, size_t pos, double *value, size_t *used)
{
  const char *begin = json.c_str() + pos;
  char *end = nullptr;
  *value = std::strtod(begin, &end);
  *used = static_cast<size_t>(end - begin);
  return *used > 0 && std::isfinite(*value);
}

bool LaxDouble(const std::string &json, const std::string &key, double *value)
{
  size_t pos = 0, used = 0;
  return ValueStart(json, key, &pos) && Number(json, pos, value, &used);
}

bool LaxDoubleArray(const std::string &json, const std::string &key, std::vector<double> *values)
{
  size_t pos = 0;
  if (!ValueStart(json, key, &pos) || json[pos] != '[')
    return false;
  ++pos;
  values->clear();
  auto skip = [&] {
    while (pos < json.size() && std::isspace(static_cast<unsigned char>(json[pos])))
      ++pos;
  };
  while (pos < json.size()) {
    skip();
    if (pos >= json.size())
      return false;
    if (json[pos] == ']')
      return true;
    double v = 0.0;
    size_t used = 0;
    if (!Number(json, pos, &v, &used))
      return false;
    values->push_back(v);
    pos += used;
    skip();
    if (pos >= json.size() || (json[pos] != ',' && json[pos] != ']'))
      return false;
    if (json[pos] == ']')
      return true;
    ++pos;
  }
  return false;
}

// P1 area and the curl basis (BuildElementTerms); false for a non-positive area.
bool Area(const double *p0, const double *p1, const double *p2, double *area)
{
  const double det = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
  *area = 0.5 * det;
  return std::isfinite(det) && det > 0.0;
}

} // namespace

bool ParseSingleSampleRequestText(const std::string &json, SingleSampleRequest *r, std::string *error)
{
  std::string protocol;
  double selected = 0.0;
  if (!LaxString(json, "protocol", &protocol) || protocol != "gpu_femm_single_sample_v1" ||
      !LaxString(json, "stem", &r->stem) || !LaxString(json, "curve_directory", &r->curve_directory) ||
      !LaxString(json, "source_motor_fem_sha256", &r->source_motor_fem_sha256) ||
      !LaxDouble(json, "current_A", &r->current_a) || !LaxDouble(json, "selected_material_label", &selected) ||
      !LaxDouble(json, "airgap_radius_mm", &r->airgap_radius_mm) ||
      !LaxDoubleArray(json, "airgap_angles_deg", &r->airgap_angles_deg) || r->stem.empty() ||
      r->curve_directory.empty() || r->source_motor_fem_sha256.size() != 64 || !(r->airgap_radius_mm >= 0.0) ||
      (!r->airgap_angles_deg.empty() && !(r->airgap_radius_mm > 0.0))) {
    *error = "invalid gpu_femm_single_sample_v1 request";
    return false;
  }
  // The label is converted like a C++ static_cast; the value must be exactly 1.
  if (!(selected >= -2147483648.0 && selected < 2147483648.0) || selected != std::trunc(selected) ||
      selected != 1.0) {
    *error = "frozen adapter requires selected_material_label=1";
    return false;
  }
  r->selected_material_label = 1;
  for (unsigned char c : r->source_motor_fem_sha256)
    if (!std::isxdigit(c)) {
      *error = "source_motor_fem_sha256 must be hexadecimal";
      return false;
    }
  return true;
}

bool ReadFemmNonlinear(const std::string &stem, const std::string &curve_directory, Artifact *out,
                       std::vector<double> *expected_a, std::string *error)
{
  Artifact a;
  std::ifstream in(stem + ".ans");
  std::string line;
  while (std::getline(in, line) && line != "[Solution]") {
  }
  int n = 0;
  if (!in || !(in >> n) || n <= 0) {
    *error = "invalid nonlinear [Solution] node count";
    return false;
  }
  a.xy.resize(2 * static_cast<size_t>(n));
  expected_a->assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    int ignored = 0;
    if (!(in >> a.xy[2 * i] >> a.xy[2 * i + 1] >> (*expected_a)[i] >> ignored)) {
      *error = "invalid nonlinear solution node";
      return false;
    }
    a.xy[2 * i] *= 1e-3;
    a.xy[2 * i + 1] *= 1e-3;
  }
  int e_count = 0;
  if (!(in >> e_count) || e_count <= 0) {
    *error = "invalid nonlinear solution element count";
    return false;
  }
  a.tri.resize(3 * static_cast<size_t>(e_count));
  a.tri_mat.resize(e_count);
  bool seen[4] = {false, false, false, false};
  std::vector<bool> boundary(n, false);
  for (int e = 0; e < e_count; ++e) {
    int edge[3] = {-1, -1, -1}, label = -1;
    double current = 0.0;
    if (!(in >> a.tri[3 * e] >> a.tri[3 * e + 1] >> a.tri[3 * e + 2] >> label >> edge[0] >> edge[1] >> edge[2] >>
          current) ||
        label < 0 || label > 3 || !std::isfinite(current)) {
      *error = "missing or out-of-range nonlinear block label";
      return false;
    }
    a.tri_mat[e] = label;
    seen[label] = true;
    for (int side = 0; side < 3; ++side)
      if (edge[side] >= 0) {
        const int p = a.tri[3 * e + side], q = a.tri[3 * e + (side + 1) % 3];
        if (p < 0 || p >= n || q < 0 || q >= n) {
          *error = "nonlinear boundary node out of range";
          return false;
        }
        boundary[p] = boundary[q] = true;
      }
  }
  for (bool s : seen)
    if (!s) {
      *error = "nonlinear fixture is missing an expected material region";
      return false;
    }
  double coil_area = 0.0;
  for (int e = 0; e < e_count; ++e) {
    const int *t = &a.tri[3 * e];
    for (int l = 0; l < 3; ++l)
      if (t[l] < 0 || t[l] >= n) {
        *error = "invalid nonlinear element geometry";
        return false;
      }
    double area = 0.0;
    if (!Area(&a.xy[2 * t[0]], &a.xy[2 * t[1]], &a.xy[2 * t[2]], &area)) {
      *error = "invalid nonlinear element geometry";
      return false;
    }
    if (a.tri_mat[e] == 2)
      coil_area += area;
  }
  if (!(coil_area > 0.0)) {
    *error = "nonlinear fixture has no coil material";
    return false;
  }
  // The B-H table: a header naming both columns, then H B pairs to the end of the file.
  {
    std::ifstream table(curve_directory + "/35PN230.tab");
    std::string header;
    std::vector<double> b, h;
    if (!table || !std::getline(table, header) || header.find("H (A_per_meter)") == std::string::npos ||
        header.find("B (tesla)") == std::string::npos) {
      *error = "cannot read 35PN230 B-H table";
      return false;
    }
    double hv = 0.0, bv = 0.0;
    while (table >> hv >> bv) {
      h.push_back(hv);
      b.push_back(bv);
    }
    if (!table.eof() || b.empty()) {
      *error = "cannot read 35PN230 B-H table";
      return false;
    }
    a.curve_b = {b};
    a.curve_h = {h};
  }
  fg_material steel{1.0, 0.0, 0.0, 0.0, 0.0, 0, -1, -1, 0};
  fg_material magnet{1.0 / (kMu0 * 1.05), 0.0, 0.0, 900000.0, 0.0, -1, -1, -1, 0};
  fg_material coil{1.0 / kMu0, 0.0, 50.0 / coil_area, 0.0, 0.0, -1, 0, -1, 0};
  fg_material air{1.0 / kMu0, 0.0, 0.0, 0.0, 0.0, -1, -1, -1, 0};
  a.materials = {steel, magnet, coil, air};
  a.group_numbers = {-1, -1, -1, -1};
  a.depth_m = 0.020;
  a.problem_type = FG_PLANAR;
  for (int i = 0; i < n; ++i)
    if (boundary[i]) {
      if ((*expected_a)[i] != 0.0) {
        *error = "fixture requires zero-A outer boundary";
        return false;
      }
      a.dir_nodes.push_back(i);
      a.dir_values.push_back(0.0);
    }
  // The summary's circuit current and flux linkage must read as finite numbers when present.
  std::ifstream summary(stem + ".summary.txt");
  while (std::getline(summary, line)) {
    const size_t eq = line.find('=');
    if (eq == std::string::npos)
      continue;
    const std::string key = line.substr(0, eq);
    if (key != "circuit_current_A" && key != "flux_linkage_Wb")
      continue;
    const char *s = line.c_str() + eq + 1;
    char *end = nullptr;
    const double v = std::strtod(s, &end);
    if (end == s || !std::isfinite(v)) {
      *error = "invalid nonlinear fixture summary";
      return false;
    }
  }
  a.circuit_currents = {0.0};
  *out = std::move(a);
  return true;
}

} // namespace fgio
