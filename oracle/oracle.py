"""ctypes access to the CPU oracle and to the reference-source build.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the checker or the timed CPU path.
The product never imports this module.

* ``lib()``  -> oracle/_build/libfemm_oracle.so, the C restatement (femm_oracle.c)
* ``ref()``  -> oracle/_ref/libfemm_ref.so, FEMM-GPU's own host sources compiled here
  plus FEMM 4.2's CPU sparse PCG (fkn/spars.cpp); None when it was never built.

Models are any object with the fields of ``femm_gpu_b200.model.Model``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None


class OrModel(C.Structure):
    _fields_ = [
        ("problem_type", C.c_int32), ("node_count", C.c_int32), ("xy", C.c_void_p),
        ("tri_count", C.c_int32), ("tri", C.c_void_p), ("tri_mat", C.c_void_p),
        ("mat_count", C.c_int32), ("nu0", C.c_void_p), ("alpha", C.c_void_p),
        ("j_per_a", C.c_void_p), ("hc", C.c_void_p), ("mag_deg", C.c_void_p),
        ("curve_index", C.c_void_p), ("circuit_index", C.c_void_p),
        ("curve_count", C.c_int32), ("curve_offsets", C.c_void_p), ("curve_b", C.c_void_p),
        ("curve_h", C.c_void_p), ("dir_count", C.c_int32), ("dir_nodes", C.c_void_p),
        ("dir_values", C.c_void_p), ("con_count", C.c_int32), ("con_a", C.c_void_p),
        ("con_b", C.c_void_p), ("con_sign", C.c_void_p), ("circuit_count", C.c_int32),
        ("depth_m", C.c_double),
    ]


class OrOptions(C.Structure):
    _fields_ = [
        ("relative_tolerance", C.c_double), ("max_newton_iterations", C.c_int32),
        ("max_linear_iterations", C.c_int32), ("linear_relative_tolerance", C.c_double),
        ("recover_nonconvergence", C.c_int32), ("adaptive_linear_tolerance", C.c_int32),
    ]


class OrInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int32), ("residual_l2", C.c_double),
        ("linear_iterations", C.c_int32), ("last_linear_tolerance", C.c_double),
        ("verified_equation_residual_relative", C.c_double),
    ]


def production_options(**overrides) -> OrOptions:
    """ProductionSampleOptions (gpu_solver/src/physics/nonlinear_model.cpp:195-205)."""
    values = dict(relative_tolerance=1e-8, max_newton_iterations=128,
                  max_linear_iterations=16384, linear_relative_tolerance=1e-10,
                  recover_nonconvergence=1, adaptive_linear_tolerance=1)
    values.update(overrides)
    return OrOptions(**values)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "libfemm_oracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.or_pcg.restype = C.c_int
        _LIB.or_system_rows.restype = C.c_int32
        _LIB.or_system_nnz.restype = C.c_int32
    return _LIB


def ref():
    """The reference-source build, or None if oracle/_ref was never built here."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libfemm_ref.so")
        if not os.path.exists(path):
            return None
        _REF = C.CDLL(path)
        for name in ("ref_system_rows", "ref_system_nnz", "ref_prepared_rows", "ref_prepared_nnz",
                     "ref_prepared_matrix_entries", "ref_prepared_rhs_entries"):
            getattr(_REF, name).restype = C.c_int32
        _REF.ref_artifact_error.restype = C.c_char_p
    return _REF


class ModelView:
    """Keeps the numpy buffers alive while the C structure points at them."""

    def __init__(self, model):
        self.model = model
        offsets, cb, ch = model.curve_arrays()
        self.keep = [offsets, cb, ch]
        self.s = OrModel(
            problem_type=model.problem_type, node_count=model.node_count, xy=_p(model.xy),
            tri_count=model.tri_count, tri=_p(model.tri), tri_mat=_p(model.tri_mat),
            mat_count=model.mat_count, nu0=_p(model.nu0), alpha=_p(model.alpha),
            j_per_a=_p(model.j_per_a), hc=_p(model.hc), mag_deg=_p(model.mag_deg),
            curve_index=_p(model.curve_index), circuit_index=_p(model.circuit_index),
            curve_count=len(model.curves), curve_offsets=_p(offsets), curve_b=_p(cb),
            curve_h=_p(ch), dir_count=int(model.dir_nodes.size), dir_nodes=_p(model.dir_nodes),
            dir_values=_p(model.dir_values), con_count=int(model.con_a.size),
            con_a=_p(model.con_a), con_b=_p(model.con_b), con_sign=_p(model.con_sign),
            circuit_count=model.circuit_count, depth_m=model.depth_m)

    def ref(self):
        return C.byref(self.s)


def bh_build(b, h, use_ref=False):
    b = np.array(b, dtype=np.float64)
    h = np.array(h, dtype=np.float64)
    slope = np.zeros_like(b)
    cold = C.c_double(0.0)
    passes = C.c_int32(0)
    fn = ref().ref_bh_build if use_ref else lib().or_bh_build
    ok = fn(C.c_int32(b.size), _p(b), _p(h), _p(slope), C.byref(cold), C.byref(passes))
    if not ok:
        raise ValueError("invalid B-H curve")
    return b, h, slope, cold.value, passes.value


def bh_eval(b, h, slope, field_b, use_ref=False):
    out = np.zeros(4)
    fn = ref().ref_bh_eval if use_ref else lib().or_bh_eval
    fn(C.c_int32(b.size), _p(b), _p(h), _p(slope), C.c_double(field_b), _p(out))
    return out


class System:
    """A reduced Newton system (CSR, diagonal, rhs, node maps)."""

    def __init__(self, rows, off, col, val, diag, rhs, node_to_free, node_sign, boundary, sources=None):
        self.rows, self.off, self.col, self.val = rows, off, col, val
        self.diag, self.rhs, self.node_to_free = diag, rhs, node_to_free
        self.node_sign, self.boundary, self.sources = node_sign, boundary, sources


def assemble(model, a_old, currents, use_newton, use_ref=False) -> System:
    view = ModelView(model)
    a_old = np.ascontiguousarray(a_old, dtype=np.float64)
    currents = np.ascontiguousarray(currents, dtype=np.float64)
    handle = C.c_void_p()
    if use_ref:
        r = ref()
        status = r.ref_assemble(view.ref(), _p(a_old), _p(currents), C.c_int(int(use_newton)),
                                C.byref(handle))
        if status:
            raise RuntimeError(f"reference assembly status {status}")
        rows, nnz = r.ref_system_rows(handle), r.ref_system_nnz(handle)
    else:
        o = lib()
        status = o.or_assemble(view.ref(), _p(a_old), _p(currents), C.c_int(int(use_newton)),
                               C.byref(handle))
        if status:
            raise RuntimeError(f"oracle assembly status {status}")
        rows, nnz = o.or_system_rows(handle), o.or_system_nnz(handle)
    N = model.node_count
    off = np.zeros(rows + 1, np.int32)
    col = np.zeros(nnz, np.int32)
    val = np.zeros(nnz)
    diag = np.zeros(rows)
    rhs = np.zeros(rows)
    n2f = np.zeros(N, np.int32)
    sign = np.zeros(N, np.int8)
    bnd = np.zeros(N)
    src = None
    if use_ref:
        r.ref_system_copy(handle, _p(off), _p(col), _p(val), _p(diag), _p(rhs), _p(n2f), _p(sign), _p(bnd))
        r.ref_system_free(handle)
    else:
        src = np.zeros(max(model.circuit_count, 1) * rows)
        o.or_system_copy(handle, _p(off), _p(col), _p(val), _p(diag), _p(rhs), _p(n2f), _p(sign),
                         _p(bnd), _p(src))
        o.or_system_free(handle)
        src = src[: model.circuit_count * rows].reshape(model.circuit_count, rows)
    return System(rows, off, col, val, diag, rhs, n2f, sign, bnd, src)


def pcg(system: System, rhs=None, tol=1e-10, maxit=16384):
    rhs = system.rhs if rhs is None else np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(system.rows)
    its = C.c_int32(0)
    res = C.c_double(0.0)
    status = lib().or_pcg(C.c_int32(system.rows), _p(system.off), _p(system.col), _p(system.val),
                          _p(system.diag), _p(rhs), C.c_double(tol), C.c_int32(maxit), _p(x),
                          C.byref(its), C.byref(res))
    return status, x, its.value, res.value


def set_preconditioner(kind=0, block_size=8):
    """Preconditioner of pcg() and solve_batch(): 0 Jacobi, 1 block-Jacobi (block_size rows)."""
    lib().or_set_preconditioner(C.c_int32(kind), C.c_int32(block_size))


class preconditioner:
    """with preconditioner(1, 8): ... -- block-Jacobi for the oracle calls inside."""

    def __init__(self, kind, block_size=8):
        self.kind, self.block_size = kind, block_size

    def __enter__(self):
        set_preconditioner(self.kind, self.block_size)

    def __exit__(self, *exc):
        set_preconditioner(0, 8)


def block_jacobi(system: System, bs=8):
    """Block inverses [blocks][bs*bs] (entry (i, j) at j*bs+i; NaN first entry = unusable)
    and the count of unusable blocks."""
    blocks = (system.rows + bs - 1) // bs
    inv = np.zeros(blocks * bs * bs)
    fb = C.c_int32(0)
    st = lib().or_block_jacobi(C.c_int32(system.rows), _p(system.off), _p(system.col),
                               _p(system.val), _p(system.diag), C.c_int32(bs), _p(inv), C.byref(fb))
    if st:
        raise RuntimeError(f"or_block_jacobi status {st}")
    return inv.reshape(blocks, bs * bs), fb.value


def csr_system(off, col, val, rhs=None):
    """A System view of caller CSR arrays (diagonal taken from the entries)."""
    sysm = System.__new__(System)
    sysm.off = np.ascontiguousarray(off, dtype=np.int32)
    sysm.col = np.ascontiguousarray(col, dtype=np.int32)
    sysm.val = np.ascontiguousarray(val, dtype=np.float64)
    sysm.rows = sysm.off.size - 1
    diag = np.zeros(sysm.rows)
    for r in range(sysm.rows):
        for k in range(sysm.off[r], sysm.off[r + 1]):
            if sysm.col[k] == r:
                diag[r] = sysm.val[k]
    sysm.diag = diag
    sysm.rhs = None if rhs is None else np.ascontiguousarray(rhs, dtype=np.float64)
    return sysm


def solve_batch(model, currents, options=None, warm=None):
    """Reference Newton semantics for a batch of circuit-current vectors."""
    currents = np.ascontiguousarray(np.atleast_2d(currents), dtype=np.float64)
    k = currents.shape[0]
    view = ModelView(model)
    N, E, Cc = model.node_count, model.tri_count, model.circuit_count
    a = np.zeros((k, N))
    b1 = np.zeros((k, E))
    b2 = np.zeros((k, E))
    flux = np.zeros((k, max(Cc, 1)))
    info = (OrInfo * k)()
    opts = options if options is not None else production_options()
    warm_arr = None if warm is None else np.ascontiguousarray(warm, dtype=np.float64)
    lib().or_solve_batch(view.ref(), C.c_int32(k), _p(currents), _p(warm_arr), C.byref(opts),
                         _p(a), _p(b1), _p(b2), _p(flux), info)
    return a, b1, b2, flux[:, :Cc], [info[i] for i in range(k)]


def signed_dofs(node_count, con_a, con_b, con_sign, dir_nodes, dir_values):
    root = np.zeros(node_count, np.int32)
    sign = np.zeros(node_count, np.int8)
    n2f = np.zeros(node_count, np.int32)
    bnd = np.zeros(node_count)
    nf = C.c_int32(0)
    arrs = [np.ascontiguousarray(con_a, np.int32), np.ascontiguousarray(con_b, np.int32),
            np.ascontiguousarray(con_sign, np.int8), np.ascontiguousarray(dir_nodes, np.int32),
            np.ascontiguousarray(dir_values, np.float64)]
    rc = lib().or_signed_dofs(C.c_int32(node_count), C.c_int32(arrs[0].size), _p(arrs[0]), _p(arrs[1]),
                              _p(arrs[2]), C.c_int32(arrs[3].size), _p(arrs[3]), _p(arrs[4]),
                              _p(root), _p(sign), _p(n2f), _p(bnd), C.byref(nf))
    return rc, root, sign, n2f, bnd, nf.value


def validate(model, use_ref=False):
    view = ModelView(model)
    if use_ref:
        return ref().ref_validate(view.ref())
    return lib().or_validate(view.ref())


def ref_cpu_newton_batch(model, currents, options=None, threads=1):
    """Reference host assembler + FEMM CBigLinProb PCG (SSOR) Newton solves on host threads."""
    r = ref()
    if r is None:
        raise RuntimeError("oracle/_ref/libfemm_ref.so not built")
    currents = np.ascontiguousarray(np.atleast_2d(currents), dtype=np.float64)
    k = currents.shape[0]
    view = ModelView(model)
    N, Cc = model.node_count, model.circuit_count
    a = np.zeros((k, N))
    flux = np.zeros((k, Cc))
    status = np.zeros(k, np.int32)
    newton = np.zeros(k, np.int32)
    calls = np.zeros(k, np.int32)
    worst = np.zeros(k)
    opts = options if options is not None else production_options()
    rc = r.ref_cpu_newton_batch(view.ref(), C.c_int32(k), _p(currents), C.byref(opts),
                                C.c_int32(threads), _p(a), _p(flux), _p(status), _p(newton),
                                _p(calls), _p(worst))
    if rc:
        raise RuntimeError(f"reference CPU baseline status {rc}")
    return a, flux, status, newton, calls, worst


class RefSession:
    """Step-wise reference CPU path: k samples, each step = one Newton iteration of every
    unfinished sample (host assembly + FEMM PCG), one sample per host thread."""

    def __init__(self, model, currents, options=None):
        r = ref()
        if r is None:
            raise RuntimeError("oracle/_ref/libfemm_ref.so not built")
        self.r = r
        r.ref_session_create.restype = C.c_int32
        r.ref_session_destroy.restype = None
        self.view = ModelView(model)
        currents = np.ascontiguousarray(np.atleast_2d(currents), dtype=np.float64)
        self.k, self.c = currents.shape
        self.opts = options if options is not None else production_options()
        self.handle = C.c_void_p()
        rc = r.ref_session_create(self.view.ref(), C.c_int32(self.k), _p(currents),
                                  C.byref(self.opts), C.byref(self.handle))
        if rc:
            raise RuntimeError(f"reference session status {rc}")
        self.done = np.zeros(self.k, np.int32)

    def step(self, threads):
        self.r.ref_session_step(self.handle, C.c_int32(threads), _p(self.done))
        return self.done.copy()

    def restart(self, i, currents):
        cur = np.ascontiguousarray(currents, dtype=np.float64)
        self.r.ref_session_restart(self.handle, C.c_int32(i), _p(cur))
        self.done[i] = 0

    def info(self):
        status = np.zeros(self.k, np.int32)
        newton = np.zeros(self.k, np.int32)
        self.r.ref_session_info(self.handle, _p(status), _p(newton))
        return status, newton

    def close(self):
        if self.handle:
            self.r.ref_session_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        self.close()
