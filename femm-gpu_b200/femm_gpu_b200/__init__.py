"""femm_gpu_b200: Python host side of libfemmgpu, the B200 nonlinear magnetostatic solver.

* ``Model`` -- the in-memory model crossing the C ABI (mirrors FEMM-GPU's NonlinearModel)
* ``Plan`` -- fg_plan_create / fg_solve_batch / ... over ctypes
* ``meshes`` -- seeded synthetic workloads
* ``artifact`` -- the gpu_femm_magnetostatic_mesh_v1 JSON artifact writer
"""
from . import meshes
from .capi import (Plan, Multi, Postprocess, SolveResult, FgError, csr_pcg, lib, production_options,
                   status_name, bh_build, bh_eval, LIB_PATH, STATUS_NAMES, EXPORTED)
from .model import AXISYMMETRIC, MU0, PLANAR, AirGap, Model

__all__ = ["Model", "AirGap", "Plan", "Multi", "Postprocess", "SolveResult", "FgError", "csr_pcg", "lib",
           "production_options", "status_name", "bh_build", "bh_eval", "meshes", "LIB_PATH", "STATUS_NAMES", "EXPORTED",
           "PLANAR", "AXISYMMETRIC", "MU0"]
