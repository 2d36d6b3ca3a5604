// artifact.h -- gpu_femm_magnetostatic_mesh_v1 / gpu_femm_planar_dc_mesh_v1 mesh artifacts.
#pragma once

#include "femm_gpu.h"
#include "json.h"

#include <string>
#include <vector>

namespace fgio
{

// One native air-gap element of a sliding-band artifact (AirGapElement as
// ParseGpuFemmMeshArtifactJson maps it, io/mesh_artifact.cpp:633-696): millimetres to
// metres, per band point the inner-ring pair n0 / n1 and the outer-ring pair n2 / n3 with
// their copy signs.
struct AirGapBand {
  std::string name;
  bool antiperiodic = false;
  double center_m[2] = {0.0, 0.0}, ri_m = 0.0, ro_m = 0.0, arc_deg = 0.0;
  double inner_shift = 0.0, outer_shift = 0.0;
  int32_t sector_count = 0;
  std::vector<int32_t> nodes;  // [4 * (sector_count + 1)]
  std::vector<double> weights; // [4 * (sector_count + 1)]
};

// A parsed artifact owning every array an fg_model points at.
struct Artifact {
  std::string schema_version, source_fem_sha256, canonical_identity_sha256;
  // Motor schema (gpu_femm_mesh_v1): the base motor identity and the mesh's pose.
  bool motor = false;
  std::string base_motor_fem_sha256;
  double rotor_angle_deg = 0.0, displacement_mm[2] = {0.0, 0.0};
  // gpu_femm_mesh_v3: a conforming 180-degree sector and how the full machine follows.
  bool sector = false;
  double sector_start_angle_deg = 0.0, sector_angle_deg = 0.0;
  int32_t full_machine_sector_count = 0, electrical_pole_pairs = 0, suspension_spatial_order = 0;
  int32_t sector_boundary_sign = 1;
  std::string model_invariance_certificate_sha256;
  std::vector<int32_t> apex_nodes; // rotational apex self-pairs (origin nodes)
  std::vector<int32_t> circuit_partners;
  std::vector<int8_t> circuit_orientations;
  int32_t problem_type = FG_PLANAR;
  double depth_m = 0.0;
  std::vector<double> xy;
  std::vector<int32_t> tri, tri_mat;
  std::vector<fg_material> materials;
  std::vector<std::vector<double>> curve_b, curve_h;
  std::vector<fg_bh_curve> curves;
  std::vector<int32_t> dir_nodes;
  std::vector<double> dir_values;
  std::vector<int32_t> con_nodes;
  std::vector<int8_t> con_signs;
  std::vector<double> circuit_currents;
  std::vector<int32_t> group_numbers; // per expanded label material
  // gpu_femm_mesh_v2: a zero-degree reference mesh whose air gap is native air-gap elements;
  // each rotor angle is a pose of the bands (SlideBands), not a new mesh.
  bool sliding_band = false;
  bool native_sector = false; // gpu_femm_mesh_v4: a cyclic sector whose air gap is native elements
  std::vector<AirGapBand> bands;
  std::vector<fg_air_gap_element> band_view; // filled by Model()

  // The fg_model view (valid while this object lives and is not modified).
  fg_model Model();
  // ApplySlidingBandAngle (io/sample_request.cpp:448-491): poses the bands of this
  // zero-degree artifact at rotor_angle_deg.  The inner ring slides by the angle over the
  // band's arc: the whole arcs rotate the inner records cyclically (the last point repeats
  // the first), the fraction becomes the new inner shift; the stator side stays.  False for
  // a non-finite angle or a degenerate band.
  bool SlideBands(double rotor_angle_deg);
};

// ParseGpuFemmMeshArtifactJson (gpu_solver/src/io/mesh_artifact.cpp:14-715) for the two
// neutral schemas and the conforming posed motor schema gpu_femm_mesh_v1: the same
// acceptance rules and the same mapping -- millimetres to metres, nu0 = 1 / (mu0 mu_x), one
// label material per region appended after the base materials (group, circuit, magnet
// angle, J = turns / region area), zero outer Dirichlet values, signed node constraints.
// and its conforming 180-degree sector gpu_femm_mesh_v3 (sector metadata, apex self-pairs,
// circuit partners), and the sliding-band schema gpu_femm_mesh_v2 (a zero-degree reference
// mesh with native air-gap elements) and its cyclic sector gpu_femm_mesh_v4 (one of k
// sectors with a native air-gap element band over the sector).
bool ParseArtifact(const std::string &text, Artifact *out, std::string *error);

} // namespace fgio
