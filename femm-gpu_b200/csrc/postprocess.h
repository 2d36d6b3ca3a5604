// postprocess.h -- frozen-state postprocessing: weighted-stress force / torque on a selected
// region and FEMM-smoothed radial air-gap flux density (gpu_solver/src/postprocess/).
#pragma once

#include "common.h"
#include "femm_gpu.h"
#include "model.h"

#include <cstdint>
#include <vector>

namespace fg
{

// One air-gap probe: the first containing element in element order and its barycentric
// coordinates (FrozenAirgapProbe, postprocess.h:45-50 of the reference).
struct AirgapProbe {
  int32_t element = -1;
  double lambda[3] = {};
  double cosine = 0.0, sine = 0.0;
};

// FEMM's nodal B at one probe corner as a fixed recipe: which elements and nodes the
// smoothing reads, in which order, with which weights -- all set by the mesh and its labels.
// kind 0: centroid-distance average over terms (element, w); 1: interface traversal over
// terms (source element, other node, w, tangent, length); 2: mesh edge, B of `element`;
// 3: an interface corner replaced by the sharp-corner fallback (the largest |B| among the
// corner's same-label elements, listed in terms, along B of `element`); -1: the smoothing
// fails for every solution (MESH_INVALID).
struct CornerStencil {
  int32_t kind, first, count, element, node, reserved;
  double wsum;
};

// The reusable, solution-independent part (FrozenPostprocessPlan, postprocess.h:52-70).
struct PostprocessPlan {
  std::vector<double> mask;            // [N] 0 / 1
  std::vector<double> hx, hy;          // [E] mask gradient (curl form)
  std::vector<double> weight;          // [E] area * depth
  std::vector<double> cx, cy;          // [E] centroids
  std::vector<std::vector<int32_t>> incident; // node -> elements, element order
  std::vector<AirgapProbe> probes;
  // The device form's smoothing recipes: corners [3 * probes], their terms.
  std::vector<CornerStencil> corners;
  std::vector<int32_t> term_elem, term_node;
  std::vector<double> term_w, term_tx, term_ty, term_len;
};

// PrepareWeightedStressMask + SolveWeightedStressMask (weighted_stress.cu:24-183), the
// linear solve on the GPU through fg_csr_pcg.
Status WeightedStressMask(const HostModel &model, const fg_postprocess_options &options,
                          std::vector<double> *mask);
// BuildFrozenPostprocessPlanWithMask (field_postprocess.cpp:221-339).
Status BuildPostprocessPlan(const HostModel &model, const fg_postprocess_options &options,
                            std::vector<double> mask, PostprocessPlan *plan);
// ComputeFrozenPostprocess (field_postprocess.cpp:341-403) for one solution; radial_b
// [probes].  Returns the item's status.
Status ComputePostprocess(const HostModel &model, const PostprocessPlan &plan, const double *a,
                          const double *b1, const double *b2, fg_postprocess_result *result,
                          double *radial_b);

// ComputeFrozenTangentPostprocess (field_postprocess.cpp:405-520) with the reusable plan:
// force / torque / radial B derivatives of one tangent solution about base B.
Status ComputeTangentPostprocess(const HostModel &model, const PostprocessPlan &plan, const double *base_b1,
                                 const double *base_b2, const double *da, const double *db1,
                                 const double *db2, fg_postprocess_result *result, double *radial_b);

// Device form: force / torque partial sums per (CTA, item) and the air-gap samples of every
// (item, probe) from the corner recipes, in one launch.
struct PostprocessDevice {
  const double *hx, *hy, *weight, *cx, *cy; // [E]
  const CornerStencil *corners;             // [3 * probes]
  const int32_t *term_elem, *term_node;
  const double *term_w, *term_tx, *term_ty, *term_len;
  const double *probe;                      // [probes][5]: lambda 0..2, cos, sin
  int32_t E, N, items, ctas, probes;
  const double *a, *b1, *b2; // item-major solutions
  double *partials;          // [ctas][items][3]
  double *radial;            // [items][probes]
};
int PostprocessCtas(int32_t E, int32_t items);
cudaError_t LaunchPostprocess(const PostprocessDevice &p, cudaStream_t stream);

} // namespace fg

struct fg_postprocess {
  fg::HostModel model; // geometry and labels only
  fg::PostprocessPlan plan;
  // Device copies (created by the first fg_postprocess_compute_device).
  fg::DeviceArray<double> geometry; // hx, hy, weight, cx, cy [5][E]; probes [5P]; terms w, tx, ty, len
  fg::DeviceArray<int32_t> terms;   // term_elem, term_node
  fg::DeviceArray<fg::CornerStencil> corners;
  fg::DeviceArray<double> out;      // partials, radial
  fg::PinnedArray<double> host_out;
};
