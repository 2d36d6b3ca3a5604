// femm_ans.h -- the frozen single-sample adapter's inputs: the gpu_femm_single_sample_v1
// request and FEMM 4.2 .ans nonlinear PM / coil solutions.
#pragma once

#include "artifact.h"

#include <string>
#include <vector>

namespace fgio
{

// gpu_femm_single_sample_v1 (ReadSingleSampleRequest, gpu_solver/src/io/sample_request.cpp:
// 98-135): the reference reads it with key-search helpers, not the strict parser -- the
// first occurrence of "key" anywhere in the text, then ':' and the value; strings end at
// the next quote and may not hold a backslash; numbers are strtod prefixes.  The same
// reading rules apply here.
struct SingleSampleRequest {
  std::string stem, curve_directory, source_motor_fem_sha256;
  double current_a = 0.0;
  int32_t selected_material_label = 0;
  double airgap_radius_mm = 0.0;
  std::vector<double> airgap_angles_deg;
};

bool ParseSingleSampleRequestText(const std::string &text, SingleSampleRequest *out, std::string *error);

// ReadNonlinearFemmReference (gpu_solver/tests/native/reference.cpp:229-379): nodes (mm)
// and P1 elements of the [Solution] section of stem.ans, block labels 0..3 mapped onto the
// fixture's materials (0 Steel35PN230 with the B-H table curve_directory/35PN230.tab,
// 1 linear PM mu_r 1.05 and Hc 900 kA/m along +x, 2 coil air driven by circuit 0 with 50
// turns over the label-2 area, 3 air), zero Dirichlet values on every node of a boundary
// edge, depth 20 mm, one circuit.  `expected_a` receives FEMM's nodal A.
bool ReadFemmNonlinear(const std::string &stem, const std::string &curve_directory, Artifact *out,
                       std::vector<double> *expected_a, std::string *error);

} // namespace fgio
