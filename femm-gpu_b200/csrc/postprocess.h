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

// The reusable, solution-independent part (FrozenPostprocessPlan, postprocess.h:52-70).
struct PostprocessPlan {
  std::vector<double> mask;            // [N] 0 / 1
  std::vector<double> hx, hy;          // [E] mask gradient (curl form)
  std::vector<double> weight;          // [E] area * depth
  std::vector<double> cx, cy;          // [E] centroids
  std::vector<std::vector<int32_t>> incident; // node -> elements, element order
  std::vector<AirgapProbe> probes;
  // What the probes' smoothing reads: elements incident to any probe corner and the nodes
  // of those elements, ascending.
  std::vector<int32_t> gather_elements, gather_nodes;
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

// Device form: force / torque partial sums per CTA and the probe gathers in one launch.
struct PostprocessDevice {
  const double *hx, *hy, *weight, *cx, *cy; // [E]
  const int32_t *gather_elements, *gather_nodes;
  int32_t E, N, items, ctas, gather_e, gather_n;
  const double *a, *b1, *b2; // item-major solutions
  double *partials;          // [ctas][items][3]
  double *gathered;          // [items][2 * gather_e + gather_n]
};
int PostprocessCtas(int32_t E);
cudaError_t LaunchPostprocess(const PostprocessDevice &p, cudaStream_t stream);

} // namespace fg

struct fg_postprocess {
  fg::HostModel model; // geometry and labels only
  fg::PostprocessPlan plan;
  // Device copies (created by the first fg_postprocess_compute_device).
  fg::DeviceArray<double> geometry; // hx, hy, weight, cx, cy: [5][E]
  fg::DeviceArray<int32_t> gathers; // gather_elements, gather_nodes
  fg::DeviceArray<double> out;      // partials, gathered
  fg::PinnedArray<double> host_out;
};
