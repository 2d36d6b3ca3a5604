"""Regenerates tests/golden/ from the reference checkout's own test fixtures.

Run once with the FEMM_GPU_REFERENCE environment variable naming a reference checkout.  The files are the reference's frozen
golden vectors for this path, copied byte for byte (gpu_solver/tests/fixtures/...):

* 35PN230.tab, reference_samples.txt, smoothing_reference.txt  (B-H spline / eval)
* periodic_strip.gpu.json, antiperiodic_strip.gpu.json, axisymmetric_coil.gpu.json
  and their stock-FEMM *.summary.txt flux linkages (constraint folding, r-z element)
* nonlinear_pm_coil_planar.{ans,summary.txt,postprocess.txt} and
  nonlinear_pm_coil_single_sample_request.json: FEMM 4.2's own nonlinear PM / coil
  solution with its weighted-stress force / torque and smoothed air-gap B samples
  (the --single-sample fixture)
* motor_mesh_v1.gpu.json: the reference's posed motor artifact fixture (gpu_femm_mesh_v1)

plus expected.json: the stock-FEMM flux linkages parsed from the summaries.
"""
import json
import os
import shutil

REF = os.environ.get("FEMM_GPU_REFERENCE", "")
FIX = os.path.join(REF, "gpu_solver", "tests", "fixtures")
HERE = os.path.dirname(os.path.abspath(__file__))

FILES = {
    "35PN230_v1/35PN230.tab": "35PN230.tab",
    "35PN230_v1/reference_samples.txt": "35PN230_reference_samples.txt",
    "35PN230_v1/smoothing_reference.txt": "35PN230_smoothing_reference.txt",
    "periodic_strip_v1/periodic_strip.gpu.json": "periodic_strip.gpu.json",
    "periodic_strip_v1/periodic_strip.summary.txt": "periodic_strip.summary.txt",
    "antiperiodic_strip_v1/antiperiodic_strip.gpu.json": "antiperiodic_strip.gpu.json",
    "antiperiodic_strip_v1/antiperiodic_strip.summary.txt": "antiperiodic_strip.summary.txt",
    "axisymmetric_coil_v1/axisymmetric_coil.gpu.json": "axisymmetric_coil.gpu.json",
    "axisymmetric_coil_v1/axisymmetric_coil.summary.txt": "axisymmetric_coil.summary.txt",
    "nonlinear_pm_coil_v1/nonlinear_pm_coil_planar.ans": "nonlinear_pm_coil_planar.ans",
    "nonlinear_pm_coil_v1/nonlinear_pm_coil_planar.summary.txt": "nonlinear_pm_coil_planar.summary.txt",
    "nonlinear_pm_coil_v1/nonlinear_pm_coil_planar.postprocess.txt":
        "nonlinear_pm_coil_planar.postprocess.txt",
    "nonlinear_pm_coil_v1/single_sample_request.json": "nonlinear_pm_coil_single_sample_request.json",
    "stream_worker_v1/mesh.json": "motor_mesh_v1.gpu.json",
}


def main():
    if not REF or not os.path.isdir(FIX):
        raise SystemExit("set FEMM_GPU_REFERENCE to a reference checkout (gpu_solver/tests/fixtures)")
    expected = {}
    for src, dst in FILES.items():
        shutil.copyfile(os.path.join(FIX, src), os.path.join(HERE, dst))
        if dst.endswith(".summary.txt"):
            values = dict(line.strip().split("=", 1) for line in open(os.path.join(HERE, dst))
                          if "=" in line)
            expected[dst.replace(".summary.txt", "")] = {
                "circuit_current_A": float(values["circuit_current_A"]),
                "flux_linkage_Wb": float(values["flux_linkage_Wb"]),
            }
    with open(os.path.join(HERE, "expected.json"), "w") as f:
        json.dump(expected, f, indent=2, sort_keys=True)


if __name__ == "__main__":
    main()
