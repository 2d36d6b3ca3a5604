"""ctypes binding of libfemmgpu (include/femm_gpu.h).

The library is the product: every call here goes through the C ABI into the sm_100a
kernels.  There is no CPU fallback -- if the shared library is missing or no GPU is
visible, the calls fail with an exception or a GPU_UNAVAILABLE status.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .model import Model

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libfemmgpu.so")

STATUS_NAMES = [
    "OK", "INPUT_IO", "INVALID_ARGUMENT", "UNSUPPORTED_FEATURE", "MESH_INVALID",
    "BOUNDARY_INVALID", "GPU_UNAVAILABLE", "GPU_ALLOCATION_FAILED", "ASSEMBLY_FAILED",
    "LINEAR_SOLVE_NOT_CONVERGED", "LINEAR_SOLVE_BREAKDOWN", "NUMERICAL_NONFINITE", "OUTPUT_IO",
    "INTERNAL_ERROR", "NONLINEAR_SOLVE_NOT_CONVERGED", "INVALID_MATERIAL",
]
(OK, INPUT_IO, INVALID_ARGUMENT, UNSUPPORTED_FEATURE, MESH_INVALID, BOUNDARY_INVALID,
 GPU_UNAVAILABLE, GPU_ALLOCATION_FAILED, ASSEMBLY_FAILED, LINEAR_SOLVE_NOT_CONVERGED,
 LINEAR_SOLVE_BREAKDOWN, NUMERICAL_NONFINITE, OUTPUT_IO, INTERNAL_ERROR,
 NONLINEAR_SOLVE_NOT_CONVERGED, INVALID_MATERIAL) = range(16)

PLAN_HOST_ONLY = 1
PLAN_PCG_FROM_ITERATE = 2
PLAN_PCG_ONE_REDUCTION = 4

EXPORTED = [
    "fg_production_options", "fg_status_name", "fg_abi_version", "fg_plan_create",
    "fg_plan_destroy", "fg_plan_sizes_get", "fg_plan_symbolic", "fg_assemble", "fg_pcg_solve",
    "fg_csr_pcg", "fg_solve_batch", "fg_solve_batch_device", "fg_plan_last_timing",
    "fg_bh_build", "fg_bh_eval", "fg_plan_contributors", "fg_plan_air_gap", "fg_air_gap_postprocess", "fg_air_gap_tangent", "fg_csr_pcg_noalloc",
    "fg_mlp_create", "fg_mlp_destroy", "fg_mlp_parameter_count", "fg_mlp_get_parameters",
    "fg_mlp_set_parameters", "fg_mlp_forward", "fg_mlp_loss_gradient", "fg_mlp_train",
    "fg_warm_create", "fg_warm_destroy", "fg_warm_project", "fg_warm_project_device",
    "fg_warm_predict", "fg_solve_batch_learned",
    "fg_multi_create", "fg_multi_destroy", "fg_multi_solve", "fg_multi_last_timing",
    "fg_postprocess_default_options", "fg_postprocess_create", "fg_postprocess_destroy",
    "fg_postprocess_probe_count", "fg_postprocess_mask", "fg_postprocess_compute",
    "fg_postprocess_compute_device", "fg_postprocess_frozen", "fg_postprocess_tangent",
    "fg_solve_tangent", "fg_plan_attach_device", "fg_set_wait_limit_ns", "fg_plan_pcg_shapes",
]


class FgMaterial(C.Structure):
    _fields_ = [("reluctivity_zero_m_per_h", C.c_double), ("alpha_per_t2", C.c_double),
                ("source_j_per_a", C.c_double), ("h_c_a_per_m", C.c_double),
                ("magnetization_deg", C.c_double), ("bh_curve_index", C.c_int32),
                ("circuit_index", C.c_int32), ("group_number", C.c_int32), ("reserved", C.c_int32)]


class FgCurve(C.Structure):
    _fields_ = [("count", C.c_int32), ("b_t", C.c_void_p), ("h_a_per_m", C.c_void_p)]


class FgModel(C.Structure):
    _fields_ = [
        ("problem_type", C.c_int32), ("node_count", C.c_int32), ("node_xy", C.c_void_p),
        ("triangle_count", C.c_int32), ("triangle_nodes", C.c_void_p),
        ("triangle_material", C.c_void_p), ("material_count", C.c_int32),
        ("materials", C.c_void_p), ("curve_count", C.c_int32), ("curves", C.c_void_p),
        ("dirichlet_count", C.c_int32), ("dirichlet_nodes", C.c_void_p),
        ("dirichlet_values", C.c_void_p), ("constraint_count", C.c_int32),
        ("constraint_nodes", C.c_void_p), ("constraint_signs", C.c_void_p),
        ("circuit_count", C.c_int32), ("depth_m", C.c_double),
        ("air_gap_count", C.c_int32), ("air_gap_elements", C.c_void_p),
    ]


class FgAirGap(C.Structure):
    _fields_ = [
        ("antiperiodic", C.c_int32), ("point_count", C.c_int32), ("center_x_m", C.c_double),
        ("center_y_m", C.c_double), ("inner_radius_m", C.c_double), ("outer_radius_m", C.c_double),
        ("arc_length_deg", C.c_double), ("inner_shift", C.c_double), ("outer_shift", C.c_double),
        ("nodes", C.c_void_p), ("weights", C.c_void_p),
    ]


def air_gap_array(ages):
    """ctypes fg_air_gap_element[] of Model.ages (None when there are none)."""
    if not ages:
        return None
    arr = (FgAirGap * len(ages))()
    for i, g in enumerate(ages):
        arr[i] = FgAirGap(int(bool(g.antiperiodic)), int(g.nodes.shape[0]), float(g.center_m[0]),
                          float(g.center_m[1]), float(g.inner_radius_m), float(g.outer_radius_m),
                          float(g.arc_length_deg), float(g.inner_shift), float(g.outer_shift),
                          _p(g.nodes), _p(g.weights))
    return arr


class FgPlanOptions(C.Structure):
    _fields_ = [("preconditioner", C.c_int32), ("block_size", C.c_int32),
                ("precision", C.c_int32), ("flags", C.c_int32)]


class FgSolveOptions(C.Structure):
    _fields_ = [("relative_tolerance", C.c_double), ("max_newton_iterations", C.c_int32),
                ("max_linear_iterations", C.c_int32), ("linear_relative_tolerance", C.c_double),
                ("recover_nonconvergence", C.c_int32), ("adaptive_linear_tolerance", C.c_int32)]


class FgItemInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("residual_l2", C.c_double),
                ("linear_iterations", C.c_int32), ("warm_start", C.c_int32),
                ("last_linear_tolerance", C.c_double),
                ("verified_equation_residual_relative", C.c_double)]


class FgLinearInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("residual_l2", C.c_double)]


class FgPlanSizes(C.Structure):
    _fields_ = [("node_count", C.c_int64), ("triangle_count", C.c_int64), ("rows", C.c_int64),
                ("nnz", C.c_int64), ("circuit_count", C.c_int32), ("problem_type", C.c_int32),
                ("device_bytes", C.c_int64), ("matrix_contributors", C.c_int64),
                ("rhs_contributors", C.c_int64)]


class FgTiming(C.Structure):
    _fields_ = [("assembly_ms", C.c_double), ("pcg_ms", C.c_double), ("update_ms", C.c_double),
                ("finalize_ms", C.c_double), ("newton_iterations", C.c_int64),
                ("pcg_iterations", C.c_int64), ("kernel_launches", C.c_int64),
                ("pcg_launches", C.c_int64), ("pcg_grid", C.c_int32), ("pcg_block", C.c_int32),
                ("pcg_phase_ms", C.c_double * 10), ("mixed_fallbacks", C.c_int64),
                ("block_inverses", C.c_int64), ("block_fallbacks", C.c_int64)]


class FgPcgShape(C.Structure):
    _fields_ = [("items", C.c_int32), ("precision", C.c_int32), ("block_size", C.c_int32),
                ("value_ring", C.c_int32), ("column_cache", C.c_int32), ("candidates", C.c_int32),
                ("us_per_iteration", C.c_double * 5), ("threads_per_block", C.c_int32),
                ("reserved", C.c_int32)]


_LIB = None


def build_library():
    subprocess.run(["make", "-s", "-C", PKG_DIR], check=True)


def lib():
    """Loads libfemmgpu.so (building it with nvcc first if it is absent)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build_library()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libfemmgpu.so not found at {LIB_PATH}")
        _LIB = C.CDLL(LIB_PATH)
        _LIB.fg_status_name.restype = C.c_char_p
        _LIB.fg_mlp_parameter_count.restype = C.c_int64
        _LIB.fg_mlp_destroy.restype = None
        _LIB.fg_warm_destroy.restype = None
        _LIB.fg_multi_destroy.restype = None
        _LIB.fg_postprocess_destroy.restype = None
        _LIB.fg_postprocess_default_options.restype = None
        _LIB.fg_set_wait_limit_ns.restype = C.c_int64
        _LIB.fg_set_wait_limit_ns.argtypes = [C.c_int64]
    return _LIB


def set_wait_limit_ns(ns: int) -> int:
    """fg_set_wait_limit_ns: bound of the PCG launches' grid-wide waits (ns <= 0: the
    default 5 s); returns the previous bound."""
    return int(lib().fg_set_wait_limit_ns(int(ns)))


def status_name(status: int) -> str:
    return lib().fg_status_name(int(status)).decode()


def production_options(**overrides) -> FgSolveOptions:
    o = FgSolveOptions()
    lib().fg_production_options(C.byref(o))
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class FgError(RuntimeError):
    def __init__(self, status, what=""):
        super().__init__(f"{what}: {STATUS_NAMES[status] if 0 <= status < 16 else status}")
        self.status = status


@dataclass
class SolveResult:
    a: np.ndarray  # [k, N]
    b1: np.ndarray  # [k, E]
    b2: np.ndarray  # [k, E]
    flux: np.ndarray  # [k, C]
    info: List[FgItemInfo]

    @property
    def status(self):
        return [i.status for i in self.info]


class Plan:
    """A device-resident model: fg_plan_create ... fg_plan_destroy."""

    def __init__(self, model: Model, preconditioner: int = 0, block_size: int = 8,
                 precision: int = 0, host_only: bool = False, from_iterate: bool = False,
                 one_reduction: bool = False):
        self.model = model
        L = lib()
        self._keep = []
        mats = (FgMaterial * model.mat_count)()
        for i in range(model.mat_count):
            mats[i] = FgMaterial(model.nu0[i], model.alpha[i], model.j_per_a[i], model.hc[i],
                                 model.mag_deg[i], int(model.curve_index[i]),
                                 int(model.circuit_index[i]), int(model.group[i]), 0)
        curves = (FgCurve * max(1, len(model.curves)))()
        for i, (b, h) in enumerate(model.curves):
            curves[i] = FgCurve(len(b), _p(b), _p(h))
        con = np.ascontiguousarray(np.stack([model.con_a, model.con_b], axis=1).ravel(), np.int32) \
            if model.con_a.size else np.zeros(2, np.int32)
        self._keep += [mats, curves, con]
        fm = FgModel(
            problem_type=model.problem_type, node_count=model.node_count, node_xy=_p(model.xy),
            triangle_count=model.tri_count, triangle_nodes=_p(model.tri),
            triangle_material=_p(model.tri_mat), material_count=model.mat_count,
            materials=C.cast(mats, C.c_void_p), curve_count=len(model.curves),
            curves=C.cast(curves, C.c_void_p), dirichlet_count=int(model.dir_nodes.size),
            dirichlet_nodes=_p(model.dir_nodes), dirichlet_values=_p(model.dir_values),
            constraint_count=int(model.con_a.size), constraint_nodes=_p(con),
            constraint_signs=_p(model.con_sign), circuit_count=model.circuit_count,
            depth_m=model.depth_m)
        ages = air_gap_array(model.ages)
        if ages is not None:
            self._keep.append(ages)
            fm.air_gap_count, fm.air_gap_elements = len(model.ages), C.cast(ages, C.c_void_p)
        flags = ((PLAN_HOST_ONLY if host_only else 0) | (PLAN_PCG_FROM_ITERATE if from_iterate else 0) |
                 (PLAN_PCG_ONE_REDUCTION if one_reduction else 0))
        opts = FgPlanOptions(preconditioner, block_size, precision, flags)
        self._h = C.c_void_p()
        status = L.fg_plan_create(C.byref(fm), C.byref(opts), C.byref(self._h))
        if status != 0:
            self._h = None
            raise FgError(status, "fg_plan_create")
        s = FgPlanSizes()
        L.fg_plan_sizes_get(self._h, C.byref(s))
        self.N, self.E, self.rows, self.nnz, self.C = (int(s.node_count), int(s.triangle_count),
                                                       int(s.rows), int(s.nnz), int(s.circuit_count))

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sizes(self) -> FgPlanSizes:
        s = FgPlanSizes()
        lib().fg_plan_sizes_get(self._h, C.byref(s))
        return s

    def symbolic(self):
        ro = np.zeros(self.rows + 1, np.int32)
        col = np.zeros(self.nnz, np.int32)
        n2f = np.zeros(self.N, np.int32)
        sign = np.zeros(self.N, np.int8)
        bnd = np.zeros(self.N)
        lib().fg_plan_symbolic(self._h, _p(ro), _p(col), _p(n2f), _p(sign), _p(bnd))
        return ro, col, n2f, sign, bnd

    def contributors(self):
        """Per-slot and per-row element contributor lists and the fixed PM / coil loads."""
        s = self.sizes()
        so = np.zeros(self.nnz + 1, np.int32)
        se = np.zeros((int(s.matrix_contributors), 3), np.int32)
        ro = np.zeros(self.rows + 1, np.int32)
        re = np.zeros((int(s.rhs_contributors), 3), np.int32)
        pm = np.zeros(self.rows)
        cr = np.zeros(max(self.C, 1) * self.rows)
        lib().fg_plan_contributors(self._h, _p(so), _p(se), _p(ro), _p(re), _p(pm), _p(cr))
        return so, se, ro, re, pm, cr[: self.C * self.rows].reshape(self.C, self.rows)

    def air_gap(self):
        """The fixed air-gap element terms: stiffness per CSR slot [nnz], load per row [rows]."""
        vals, rhs = np.zeros(self.nnz), np.zeros(self.rows)
        st = lib().fg_plan_air_gap(self._h, _p(vals), _p(rhs))
        if st:
            raise FgError(st, "fg_plan_air_gap")
        return vals, rhs

    def air_gap_postprocess(self, a, angles_rad=()):
        """fg_air_gap_postprocess of host nodal solutions a [k, N]: (status [k], force [k, 2],
        torque [k], radial B [k, angles])."""
        a = np.ascontiguousarray(np.atleast_2d(a), np.float64)
        k = a.shape[0]
        ang = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
        res = (FgPostprocessResult * max(k, 1))()
        radial = np.zeros((k, ang.size))
        st = lib().fg_air_gap_postprocess(self._h, C.c_int32(k), _p(a), C.c_int32(ang.size),
                                          _p(ang) if ang.size else None, res, _p(radial) if ang.size else None)
        if st:
            raise FgError(st, "fg_air_gap_postprocess")
        return PostprocessResult(status=np.array([res[i].status for i in range(k)]),
                                 force=np.array([[res[i].force_x_n, res[i].force_y_n] for i in range(k)]),
                                 torque=np.array([res[i].torque_nm for i in range(k)]), radial_b=radial)

    def air_gap_tangent(self, base_a, da, angles_rad=()):
        """fg_air_gap_tangent: derivatives along tangent solutions da [m, N] about base_a [N]."""
        base_a = np.ascontiguousarray(base_a, np.float64).ravel()
        da = np.ascontiguousarray(np.atleast_2d(da), np.float64)
        m = da.shape[0]
        ang = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
        res = (FgPostprocessResult * max(m, 1))()
        radial = np.zeros((m, ang.size))
        st = lib().fg_air_gap_tangent(self._h, C.c_int32(m), _p(base_a), _p(da), C.c_int32(ang.size),
                                      _p(ang) if ang.size else None, res, _p(radial) if ang.size else None)
        if st:
            raise FgError(st, "fg_air_gap_tangent")
        return PostprocessResult(status=np.array([res[i].status for i in range(m)]),
                                 force=np.array([[res[i].force_x_n, res[i].force_y_n] for i in range(m)]),
                                 torque=np.array([res[i].torque_nm for i in range(m)]), radial_b=radial)

    def assemble(self, states, currents, use_newton):
        states = np.ascontiguousarray(np.atleast_2d(states), np.float64)
        k = states.shape[0]
        currents = np.ascontiguousarray(np.atleast_2d(currents), np.float64).reshape(k, -1)
        un = np.ascontiguousarray(np.broadcast_to(np.asarray(use_newton, np.int32), (k,)))
        vals = np.zeros((k, self.nnz))
        diag = np.zeros((k, self.rows))
        rhs = np.zeros((k, self.rows))
        status = lib().fg_assemble(self._h, C.c_int32(k), _p(states), _p(currents), _p(un),
                                   _p(vals), _p(diag), _p(rhs))
        if status != 0:
            raise FgError(status, "fg_assemble")
        return vals, diag, rhs

    def pcg(self, values, rhs, tol=1e-10, maxit=16384, shared=False):
        rhs = np.ascontiguousarray(np.atleast_2d(rhs), np.float64)
        k = rhs.shape[0]
        values = np.ascontiguousarray(values, np.float64)
        x = np.zeros((k, self.rows))
        info = (FgLinearInfo * k)()
        status = lib().fg_pcg_solve(self._h, C.c_int32(k), _p(values),
                                    C.c_int32(0 if shared else self.nnz), _p(rhs), C.c_double(tol),
                                    C.c_int32(maxit), _p(x), info)
        if status != 0:
            raise FgError(status, "fg_pcg_solve")
        return x, [info[i] for i in range(k)]

    def solve(self, currents, hc_scale=None, warm=None, options: Optional[FgSolveOptions] = None,
              outputs=True, out: Optional[SolveResult] = None) -> SolveResult:
        """fg_solve_batch.  outputs: True (A, B, flux), "a" (A and flux only) or False (item
        info only).  out: a previous result of the same shape whose host arrays are reused
        (a serving loop's preallocated buffers)."""
        currents = np.ascontiguousarray(np.atleast_2d(np.asarray(currents, np.float64)))
        k = currents.shape[0]
        currents = currents.reshape(k, self.C) if self.C else currents
        hc = None if hc_scale is None else np.ascontiguousarray(hc_scale, np.float64)
        wm = None if warm is None else np.ascontiguousarray(warm, np.float64).reshape(k, self.N)
        opts = options if options is not None else production_options()

        def buf(name, shape, wanted):
            if not wanted:
                return None
            old = getattr(out, name, None) if out is not None else None
            if old is not None and old.shape == shape and old.dtype == np.float64 and old.flags.c_contiguous:
                return old
            return np.zeros(shape)

        a = buf("a", (k, self.N), outputs)
        b1 = buf("b1", (k, self.E), outputs is True)
        b2 = buf("b2", (k, self.E), outputs is True)
        flux = buf("_flux_full", (k, max(self.C, 1)), outputs)
        info = (FgItemInfo * k)()
        status = lib().fg_solve_batch(self._h, C.c_int32(k), _p(currents), _p(hc), _p(wm),
                                      C.byref(opts), _p(a), _p(b1), _p(b2), _p(flux), info)
        if status != 0:
            raise FgError(status, "fg_solve_batch")
        res = SolveResult(a, b1, b2, None if flux is None else flux[:, : self.C],
                          [info[i] for i in range(k)])
        res._flux_full = flux
        return res

    def solve_device(self, items, currents_ptr, options=None, hc_ptr=None, warm_ptr=None,
                     a_ptr=None, b1_ptr=None, b2_ptr=None, flux_ptr=None, stream=None):
        """Device-pointer entry (fg_solve_batch_device); pointers are integers (e.g. torch data_ptr())."""
        opts = options if options is not None else production_options()
        info = (FgItemInfo * items)()
        vp = lambda v: C.c_void_p(v) if v else None  # noqa: E731
        status = lib().fg_solve_batch_device(self._h, C.c_int32(items), vp(currents_ptr), vp(hc_ptr),
                                             vp(warm_ptr), C.byref(opts), vp(a_ptr), vp(b1_ptr),
                                             vp(b2_ptr), vp(flux_ptr), info, vp(stream))
        if status != 0:
            raise FgError(status, "fg_solve_batch_device")
        return [info[i] for i in range(items)]

    def solve_tangent(self, base_a, base_currents, directions, options: Optional[FgSolveOptions] = None):
        """Tangent multi-RHS at a converged field: returns (da [m, N], db1, db2 [m, E],
        dflux [m, C], info list)."""
        base_a = np.ascontiguousarray(base_a, np.float64).ravel()
        cur = np.ascontiguousarray(base_currents, np.float64).ravel()
        d = np.ascontiguousarray(np.atleast_2d(directions), np.float64)
        m = d.shape[0]
        opts = options if options is not None else production_options()
        da, db1, db2 = np.zeros((m, self.N)), np.zeros((m, self.E)), np.zeros((m, self.E))
        dflux = np.zeros((m, max(self.C, 1)))
        info = (FgLinearInfo * m)()
        st = lib().fg_solve_tangent(self._h, _p(base_a), _p(cur), C.c_int32(m), _p(d), C.byref(opts), _p(da),
                                    _p(db1), _p(db2), _p(dflux), info)
        if st:
            raise FgError(st, "fg_solve_tangent")
        return da, db1, db2, dflux[:, : self.C], [info[i] for i in range(m)]

    def last_timing(self) -> FgTiming:
        t = FgTiming()
        lib().fg_plan_last_timing(self._h, C.byref(t))
        return t

    def pcg_shapes(self):
        """fg_plan_pcg_shapes: the launch shapes the plan's autotuner chose, as dicts."""
        n = lib().fg_plan_pcg_shapes(self._h, 0, None)
        arr = (FgPcgShape * max(n, 1))()
        n = lib().fg_plan_pcg_shapes(self._h, n, arr)
        return [{"items": a.items, "precision": a.precision, "block_size": a.block_size,
                 "value_ring": bool(a.value_ring), "column_cache": bool(a.column_cache),
                 "candidates": a.candidates, "us_per_iteration": list(a.us_per_iteration),
                 "threads_per_block": a.threads_per_block}
                for a in arr[:n]]


def csr_pcg(row_offsets, columns, values, diagonal, rhs, tol=1e-13, maxit=64, shared=False):
    """fg_csr_pcg on an arbitrary CSR operator (values [k, nnz] or shared [nnz])."""
    ro = np.ascontiguousarray(row_offsets, np.int32)
    col = np.ascontiguousarray(columns, np.int32)
    rhs = np.ascontiguousarray(np.atleast_2d(rhs), np.float64)
    k, n = rhs.shape
    vals = np.ascontiguousarray(values, np.float64)
    diag = np.ascontiguousarray(diagonal, np.float64)
    x = np.zeros((k, n))
    info = (FgLinearInfo * k)()
    status = lib().fg_csr_pcg(C.c_int32(n), _p(ro), _p(col), _p(vals),
                              C.c_int32(0 if shared else int(ro[-1])), _p(diag), C.c_int32(k),
                              _p(rhs), C.c_double(tol), C.c_int32(maxit), _p(x), info)
    if status != 0:
        raise FgError(status, "fg_csr_pcg")
    return x, [info[i] for i in range(k)]


NOALLOC_MAX_ROWS = 16384
NOALLOC_MAX_POSITIONS = 262144


def csr_pcg_noalloc(n, row_offsets_ptr, columns_ptr, values_ptr, diagonal_ptr, rhs_ptr, x_ptr,
                    tol=1e-10, maxit=16384, stream=None):
    """fg_csr_pcg_noalloc: every pointer is a device address the caller owns (for example
    torch's ``data_ptr()``); the call itself allocates no memory.  Returns (status, info)."""
    info = FgLinearInfo()
    vp = lambda v: C.c_void_p(v) if v else None  # noqa: E731
    status = lib().fg_csr_pcg_noalloc(C.c_int32(n), vp(row_offsets_ptr), vp(columns_ptr),
                                      vp(values_ptr), vp(diagonal_ptr), vp(rhs_ptr),
                                      C.c_double(tol), C.c_int32(maxit), vp(x_ptr), C.byref(info),
                                      vp(stream))
    return status, info


def bh_build(b, h):
    b = np.array(b, np.float64)
    h = np.array(h, np.float64)
    slope = np.zeros_like(b)
    cold = C.c_double(0.0)
    passes = C.c_int32(0)
    if not lib().fg_bh_build(C.c_int32(b.size), _p(b), _p(h), _p(slope), C.byref(cold),
                             C.byref(passes)):
        raise ValueError("invalid B-H curve")
    return b, h, slope, cold.value, passes.value


def bh_eval(b, h, slope, field_b):
    out = np.zeros(4)
    lib().fg_bh_eval(C.c_int32(b.size), _p(b), _p(h), _p(slope), C.c_double(field_b), _p(out))
    return out


class FgMultiTiming(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("newton_steps", C.c_int64), ("pcg_launches", C.c_int64),
                ("graph_launches", C.c_int64), ("graph_captures", C.c_int64),
                ("kernel_launches", C.c_int64), ("max_ctas", C.c_int32), ("reserved", C.c_int32)]


class Multi:
    """fg_multi: one sample on each of several plans (meshes of any size), solved together
    with one multi-plan PCG launch per Newton step.  The plans must outlive this object."""

    def __init__(self, plans):
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[p._h for p in self.plans])
        self._h = C.c_void_p()
        st = lib().fg_multi_create(arr, C.c_int32(len(self.plans)), C.byref(self._h))
        if st:
            self._h = None
            raise FgError(st, "fg_multi_create")

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_multi_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def solve(self, currents, options: Optional[FgSolveOptions] = None, outputs=True):
        """currents: one vector per plan.  Returns (a, b1, b2, flux, info) lists."""
        M = len(self.plans)
        cur = [np.ascontiguousarray(np.asarray(c, np.float64).ravel()) for c in currents]
        a = [np.zeros(p.N) for p in self.plans] if outputs else None
        b1 = [np.zeros(p.E) for p in self.plans] if outputs is True else None
        b2 = [np.zeros(p.E) for p in self.plans] if outputs is True else None
        flux = [np.zeros(max(p.C, 1)) for p in self.plans] if outputs else None
        ptrs = lambda xs: None if xs is None else (C.c_void_p * M)(*[x.ctypes.data for x in xs])  # noqa: E731
        info = (FgItemInfo * M)()
        opts = options if options is not None else production_options()
        st = lib().fg_multi_solve(self._h, ptrs(cur), C.byref(opts), ptrs(a), ptrs(b1), ptrs(b2),
                                  ptrs(flux), info)
        if st:
            raise FgError(st, "fg_multi_solve")
        return a, b1, b2, flux, [info[i] for i in range(M)]

    def last_timing(self) -> FgMultiTiming:
        t = FgMultiTiming()
        lib().fg_multi_last_timing(self._h, C.byref(t))
        return t


class FgPostprocessOptions(C.Structure):
    _fields_ = [("selected_material_label", C.c_int32), ("air_material_label", C.c_int32),
                ("selected_group_number", C.c_int32), ("air_group_number", C.c_int32),
                ("airgap_radius_m", C.c_double), ("airgap_angle_count", C.c_int32),
                ("airgap_angles_rad", C.c_void_p), ("max_mask_iterations", C.c_int32),
                ("mask_relative_tolerance", C.c_double), ("symmetry_apex_count", C.c_int32),
                ("symmetry_apex_nodes", C.c_void_p)]


class FgPostprocessResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("reserved", C.c_int32), ("force_x_n", C.c_double),
                ("force_y_n", C.c_double), ("torque_nm", C.c_double)]


@dataclass
class PostprocessResult:
    status: np.ndarray       # [items]
    force: np.ndarray        # [items, 2] (Fx, Fy) N
    torque: np.ndarray       # [items] N m
    radial_b: np.ndarray     # [items, probes] T


class Postprocess:
    """fg_postprocess: weighted-stress force / torque on a selected region and smoothed
    radial air-gap B, reusable across the solutions of one plan.

    selected / air: material label indices, or group numbers when selected_group /
    air_group are >= 0.  mask (0 / 1 per node) skips the GPU mask solve."""

    def __init__(self, plan: Plan, selected_label=1, air_label=3, selected_group=-1, air_group=-1,
                 radius_m=0.0, angles_rad=(), max_mask_iterations=256, mask_tolerance=1e-12,
                 apex_nodes=(), mask=None):
        L = lib()
        self._angles = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
        self._apex = np.ascontiguousarray(np.asarray(apex_nodes, np.int32).ravel())
        o = FgPostprocessOptions()
        L.fg_postprocess_default_options(C.byref(o))
        o.selected_material_label, o.air_material_label = selected_label, air_label
        o.selected_group_number, o.air_group_number = selected_group, air_group
        o.airgap_radius_m = radius_m
        o.airgap_angle_count = self._angles.size
        o.airgap_angles_rad = self._angles.ctypes.data if self._angles.size else None
        o.max_mask_iterations, o.mask_relative_tolerance = max_mask_iterations, mask_tolerance
        o.symmetry_apex_count = self._apex.size
        o.symmetry_apex_nodes = self._apex.ctypes.data if self._apex.size else None
        self.options = o
        self.plan = plan
        m = None if mask is None else np.ascontiguousarray(np.asarray(mask, np.float64))
        self._h = C.c_void_p()
        st = L.fg_postprocess_create(plan._h, C.byref(o), None if m is None else _p(m), C.byref(self._h))
        if st:
            self._h = None
            raise FgError(st, "fg_postprocess_create")
        self.probes = int(L.fg_postprocess_probe_count(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().fg_postprocess_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def mask(self) -> np.ndarray:
        out = np.zeros(self.plan.N)
        st = lib().fg_postprocess_mask(self._h, _p(out))
        if st:
            raise FgError(st, "fg_postprocess_mask")
        return out

    def _result(self, res, radial):
        k = len(res)
        return PostprocessResult(
            status=np.array([res[i].status for i in range(k)]),
            force=np.array([[res[i].force_x_n, res[i].force_y_n] for i in range(k)]).reshape(k, 2),
            torque=np.array([res[i].torque_nm for i in range(k)]), radial_b=radial)

    def compute(self, a, b1, b2) -> PostprocessResult:
        """Host solutions: a [k, N], b1 / b2 [k, E]."""
        a = np.ascontiguousarray(np.atleast_2d(a), np.float64)
        b1 = np.ascontiguousarray(np.atleast_2d(b1), np.float64)
        b2 = np.ascontiguousarray(np.atleast_2d(b2), np.float64)
        k = a.shape[0]
        res = (FgPostprocessResult * max(k, 1))()
        radial = np.zeros((k, self.probes))
        st = lib().fg_postprocess_compute(self._h, C.c_int32(k), _p(a), _p(b1), _p(b2), res,
                                          _p(radial) if self.probes else None)
        if st:
            raise FgError(st, "fg_postprocess_compute")
        return self._result([res[i] for i in range(k)], radial)

    def tangent(self, base_b1, base_b2, da, db1, db2) -> PostprocessResult:
        """Derivatives about base B of tangent solutions da [m, N], db1 / db2 [m, E]."""
        b1 = np.ascontiguousarray(base_b1, np.float64).ravel()
        b2 = np.ascontiguousarray(base_b2, np.float64).ravel()
        da = np.ascontiguousarray(np.atleast_2d(da), np.float64)
        db1 = np.ascontiguousarray(np.atleast_2d(db1), np.float64)
        db2 = np.ascontiguousarray(np.atleast_2d(db2), np.float64)
        m = da.shape[0]
        res = (FgPostprocessResult * max(m, 1))()
        radial = np.zeros((m, self.probes))
        st = lib().fg_postprocess_tangent(self._h, C.c_int32(m), _p(b1), _p(b2), _p(da), _p(db1), _p(db2), res,
                                          _p(radial) if self.probes else None)
        if st:
            raise FgError(st, "fg_postprocess_tangent")
        return self._result([res[i] for i in range(m)], radial)

    def compute_device(self, k, a_ptr, b1_ptr, b2_ptr, stream=0) -> PostprocessResult:
        """Device solutions (item-major) by pointer, e.g. torch tensors' data_ptr()."""
        res = (FgPostprocessResult * max(k, 1))()
        radial = np.zeros((k, self.probes))
        st = lib().fg_postprocess_compute_device(
            self._h, C.c_int32(k), C.c_void_p(a_ptr), C.c_void_p(b1_ptr), C.c_void_p(b2_ptr), res,
            _p(radial) if self.probes else None, C.c_void_p(stream))
        if st:
            raise FgError(st, "fg_postprocess_compute_device")
        return self._result([res[i] for i in range(k)], radial)
