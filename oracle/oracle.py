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
        ("depth_m", C.c_double), ("age_count", C.c_int32), ("ages", C.c_void_p),
    ]


class OrAirGap(C.Structure):
    _fields_ = [
        ("antiperiodic", C.c_int32), ("point_count", C.c_int32), ("center_x_m", C.c_double),
        ("center_y_m", C.c_double), ("inner_radius_m", C.c_double), ("outer_radius_m", C.c_double),
        ("arc_length_deg", C.c_double), ("inner_shift", C.c_double), ("outer_shift", C.c_double),
        ("nodes", C.c_void_p), ("weights", C.c_void_p),
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
        ages = getattr(model, "ages", None) or []
        if ages:
            arr = (OrAirGap * len(ages))()
            for i, g in enumerate(ages):
                arr[i] = OrAirGap(int(bool(g.antiperiodic)), int(g.nodes.shape[0]), float(g.center_m[0]),
                                  float(g.center_m[1]), float(g.inner_radius_m), float(g.outer_radius_m),
                                  float(g.arc_length_deg), float(g.inner_shift), float(g.outer_shift),
                                  _p(g.nodes), _p(g.weights))
            self.keep.append(arr)
            self.s.age_count, self.s.ages = len(ages), C.cast(arr, C.c_void_p)

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


# ---- frozen postprocess (gpu_solver/src/postprocess/) ----

def _ref_model(handle):
    """The model behind a reference handle (ref_artifact_sizes / ref_artifact_copy)."""
    from femm_gpu_b200.model import Model
    r = ref()
    sizes = np.zeros(8, np.int32)
    depth, ptype = C.c_double(), C.c_int32()
    r.ref_artifact_sizes(handle, _p(sizes), C.byref(depth), C.byref(ptype))
    N, E, M, K, D, NC, NCIR, P = (int(v) for v in sizes)
    xy, tri, tm = np.zeros(2 * N), np.zeros(3 * E, np.int32), np.zeros(E, np.int32)
    md, mi = np.zeros(5 * M), np.zeros(3 * M, np.int32)
    cb, ch, cs = np.zeros(max(P, 1)), np.zeros(max(P, 1)), np.zeros(max(P, 1))
    dn, con, cu = np.zeros(max(D, 1), np.int32), np.zeros(3 * max(NC, 1), np.int32), np.zeros(max(NCIR, 1))
    r.ref_artifact_copy(handle, _p(xy), _p(tri), _p(tm), _p(md), _p(mi), _p(cb), _p(ch), _p(cs),
                        _p(dn), _p(con), _p(cu))
    md, mi, con = md.reshape(-1, 5), mi.reshape(-1, 3), con[: 3 * NC].reshape(-1, 3)
    # Curve boundaries: split the concatenated points where B restarts at the origin.
    starts = [i for i in range(P) if cb[i] == 0.0 and ch[i] == 0.0] + [P]
    curves = [(cb[starts[j]:starts[j + 1]].copy(), ch[starts[j]:starts[j + 1]].copy())
              for j in range(len(starts) - 1)]
    assert len(curves) == K
    return Model(xy=xy.reshape(-1, 2), tri=tri.reshape(-1, 3), tri_mat=tm, nu0=md[:, 0], alpha=md[:, 1],
                 j_per_a=md[:, 2], hc=md[:, 3], mag_deg=md[:, 4], curve_index=mi[:, 0],
                 circuit_index=mi[:, 1], group=mi[:, 2], curves=curves, dir_nodes=dn[:D],
                 dir_values=np.zeros(D), con_a=con[:, 0], con_b=con[:, 1], con_sign=con[:, 2],
                 circuit_count=NCIR, depth_m=depth.value, problem_type=ptype.value), cu[:NCIR]


class RefHandle:
    """A reference model handle (ref_artifact) freed with the object."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if self.h and _REF is not None:
            _REF.ref_artifact_free(self.h)
            self.h = None


def ref_femm_nonlinear(stem, curve_directory):
    """ReadNonlinearFemmReference: (handle, model, FEMM's nodal A, FEMM's flux linkage)."""
    r = ref()
    h = C.c_void_p()
    rc = r.ref_read_femm_nonlinear(stem.encode(), curve_directory.encode(), C.byref(h))
    handle = RefHandle(h)
    if rc:
        raise RuntimeError(r.ref_artifact_error(h).decode())
    model, _ = _ref_model(h)
    a = np.zeros(model.node_count)
    flux = C.c_double()
    r.ref_femm_expected(h, _p(a), C.byref(flux))
    return handle, model, a, flux.value


def ref_model_handle(model, apex_nodes=()):
    """A reference handle of an oracle model, block-label groups included; apex_nodes become
    the model's symmetry_apex_nodes (physics/nonlinear_model.h:96)."""
    r = ref()
    view = ModelView(model)
    h = C.c_void_p()
    groups = np.ascontiguousarray(model.group, np.int32)
    if r.ref_model_handle(view.ref(), _p(groups), C.byref(h)):
        raise RuntimeError("reference model conversion failed")
    apex = np.ascontiguousarray(np.asarray(apex_nodes, np.int32).ravel())
    if apex.size:
        r.ref_model_set_apex(h, C.c_int32(apex.size), _p(apex))
    return RefHandle(h)


def ref_postprocess(handle, a, b1, b2, selected_label=1, air_label=3, selected_group=-1, air_group=-1,
                    radius_m=0.0, angles_rad=(), max_mask_iterations=256, mask_tolerance=1e-12, mask=None,
                    node_count=None):
    """The reference's ComputeFrozenPostprocess (its mask through weighted_stress.cu with the
    oracle's CPU PCG in place of the device solve, unless `mask` is given).
    Returns (status, Fx, Fy, torque, radial [angles], mask [N])."""
    r = ref()
    a = np.ascontiguousarray(a, np.float64)
    b1 = np.ascontiguousarray(b1, np.float64)
    b2 = np.ascontiguousarray(b2, np.float64)
    labels = np.array([selected_label, air_label, selected_group, air_group], np.int32)
    angles = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
    out3 = np.full(3, np.nan)
    radial = np.zeros(max(angles.size, 1))
    mask_out = np.zeros(a.size)
    m = None if mask is None else np.ascontiguousarray(mask, np.float64)
    st = r.ref_postprocess(handle.h, _p(a), _p(b1), _p(b2), _p(labels), C.c_double(radius_m),
                           C.c_int32(angles.size), _p(angles), C.c_int32(max_mask_iterations),
                           C.c_double(mask_tolerance), None if m is None else _p(m), _p(out3), _p(radial),
                           _p(mask_out))
    return int(st), out3[0], out3[1], out3[2], radial[:angles.size], mask_out


def ref_read_single_sample_request(path):
    """ReadSingleSampleRequest: (True, fields dict) or (False, error)."""
    r = ref()
    bufs = [C.create_string_buffer(4096) for _ in range(4)]
    cur, rad = C.c_double(), C.c_double()
    sel, cnt = C.c_int32(), C.c_int32()
    ang = np.zeros(64)
    rc = r.ref_read_single_sample_request(str(path).encode(), bufs[0], bufs[1], bufs[2], C.byref(cur),
                                          C.byref(sel), C.byref(rad), C.byref(cnt), _p(ang), bufs[3])
    if rc:
        return False, bufs[3].value.decode()
    return True, dict(stem=bufs[0].value.decode(), curve_directory=bufs[1].value.decode(),
                      source_motor_fem_sha256=bufs[2].value.decode(), current_A=cur.value,
                      selected_material_label=sel.value, airgap_radius_mm=rad.value,
                      airgap_angles_deg=list(ang[:cnt.value]))


def weighted_stress_mask(model, selected, air, by_group=False, apex_nodes=()):
    """Numpy restatement of the weighted-stress mask (weighted_stress.cu:24-183): the
    sqrt(area)-weighted P1 Laplacian, fixed 1 on the selected region, 0 on other non-air
    regions and non-apex Dirichlet nodes, periodic across every constraint pair (sign +1),
    solved directly (scipy) and thresholded at 0.5.  None when the reference would refuse."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    N = model.node_count
    key = model.group[model.tri_mat] if by_group else model.tri_mat
    is_sel, is_air = key == selected, key == air
    fixed = np.full(N, np.nan)
    dn = np.asarray(model.dir_nodes)
    dn = dn[~np.isin(dn, np.asarray(apex_nodes, np.int64))]
    fixed[dn] = 0.0
    for e in range(model.tri_count):
        t = model.tri[e]
        if is_sel[e]:
            if np.any(np.isfinite(fixed[t]) & (fixed[t] != 1.0)):
                return None
            fixed[t] = 1.0
        elif not is_air[e]:
            fixed[t] = np.where(np.isfinite(fixed[t]), fixed[t], 0.0)
    p = model.xy[model.tri]
    det = ((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1])
           - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1]))
    area = 0.5 * det
    dx = np.stack([p[:, 1, 1] - p[:, 2, 1], p[:, 2, 1] - p[:, 0, 1], p[:, 0, 1] - p[:, 1, 1]], 1)
    dy = np.stack([p[:, 2, 0] - p[:, 1, 0], p[:, 0, 0] - p[:, 2, 0], p[:, 1, 0] - p[:, 0, 0]], 1)
    bx, by = dy / det[:, None], -dx / det[:, None]
    ke = (np.sqrt(area) * area)[:, None, None] * (bx[:, :, None] * bx[:, None, :] + by[:, :, None] * by[:, None, :])
    rows = np.repeat(model.tri, 3, axis=1).ravel()
    cols = np.tile(model.tri, (1, 3)).ravel()
    K = sp.csr_matrix((ke.ravel(), (rows, cols)), shape=(N, N))
    # Periodic pairs: union-find roots, fixed values propagated through the pairs.
    parent = np.arange(N)

    def root(i):
        while parent[i] != i:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i
    for a_, b_ in zip(model.con_a, model.con_b):
        ra, rb = root(a_), root(b_)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    roots = np.array([root(i) for i in range(N)])
    root_val = np.full(N, np.nan)
    for i in range(N):
        if np.isfinite(fixed[i]):
            if np.isfinite(root_val[roots[i]]) and root_val[roots[i]] != fixed[i]:
                return None
            root_val[roots[i]] = fixed[i]
    free_roots = np.unique(roots[~np.isfinite(root_val[roots])])
    value = root_val[roots]
    if free_roots.size:
        index = -np.ones(N, np.int64)
        index[free_roots] = np.arange(free_roots.size)
        P = sp.csr_matrix((np.ones(N), (np.arange(N), np.where(index[roots] >= 0, index[roots], 0))),
                          shape=(N, free_roots.size))
        P = P.multiply((index[roots] >= 0)[:, None]).tocsr()
        fixed_part = np.where(np.isfinite(value), value, 0.0)
        A = (P.T @ K @ P).tocsc()
        rhs = -(P.T @ (K @ fixed_part))
        x = spla.spsolve(A, rhs)
        value = np.where(index[roots] >= 0, x[np.maximum(index[roots], 0)], value)
    return (value > 0.5).astype(np.float64)


def ref_artifact_handle(text: bytes):
    """A reference handle of a mesh artifact parsed by the reference's own parser."""
    r = ref()
    h = C.c_void_p()
    rc = r.ref_parse_artifact(text, C.c_size_t(len(text)), C.byref(h))
    handle = RefHandle(h)
    if rc:
        raise RuntimeError(r.ref_artifact_error(h).decode())
    return handle


def finalize(model, a):
    """B and flux linkage of a nodal solution (or_finalize, nonlinear_solver.cu:16-83)."""
    view = ModelView(model)
    a = np.ascontiguousarray(a, np.float64)
    b1, b2 = np.zeros(model.tri_count), np.zeros(model.tri_count)
    flux = np.zeros(max(model.circuit_count, 1))
    st = lib().or_finalize(view.ref(), _p(a), _p(b1), _p(b2), _p(flux))
    if st:
        raise RuntimeError(f"oracle finalize status {st}")
    return b1, b2, flux[: model.circuit_count]


def tangent(model, base_a, base_currents, directions, tol=1e-13, maxit=16384):
    """Restatement of SolveTangentMultiRhs (nonlinear_solver.cu:85-172): the consistent
    Newton system at base_a (the oracle assembler), S_i = sum_c d_ic * (signed per-amp
    circuit load), the oracle PCG per direction, dA = signed free values (0 on fixed
    nodes), then B and flux of dA.  Returns (da [m, N], db1, db2 [m, E], dflux [m, C],
    [(status, iterations, residual)])."""
    s = assemble(model, base_a, base_currents, 1)
    d = np.atleast_2d(np.asarray(directions, np.float64))
    N = model.node_count
    out_a, out_b1, out_b2, out_f, infos = [], [], [], [], []
    for row in d:
        rhs = np.zeros(s.rows)
        for c, scale in enumerate(row):
            if scale != 0.0:
                rhs += scale * s.sources[c]
        st, x, its, res = pcg(s, rhs, tol=tol, maxit=maxit)
        da = np.where(s.node_to_free >= 0, s.node_sign * x[np.maximum(s.node_to_free, 0)], 0.0)
        b1, b2, fl = finalize(model, da)
        out_a.append(da)
        out_b1.append(b1)
        out_b2.append(b2)
        out_f.append(fl)
        infos.append((st, its, res))
    return np.array(out_a), np.array(out_b1), np.array(out_b2), np.array(out_f), infos


def ref_tangent_postprocess(handle, a, b1, b2, da, db1, db2, mask, selected_label=1, air_label=3,
                            selected_group=-1, air_group=-1, radius_m=0.0, angles_rad=()):
    """The reference's ComputeFrozenTangentPostprocess with the plan of `mask`.
    Returns (status, dFx, dFy, dtorque, radial [angles])."""
    r = ref()
    arrs = [np.ascontiguousarray(x, np.float64) for x in (a, b1, b2, da, db1, db2, mask)]
    labels = np.array([selected_label, air_label, selected_group, air_group], np.int32)
    angles = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
    out3 = np.full(3, np.nan)
    radial = np.zeros(max(angles.size, 1))
    st = r.ref_tangent_postprocess(handle.h, *[_p(x) for x in arrs[:6]], _p(labels), C.c_double(radius_m),
                                   C.c_int32(angles.size), _p(angles), _p(arrs[6]), _p(out3), _p(radial))
    return int(st), out3[0], out3[1], out3[2], radial[:angles.size]


def age_matrix(K, Ki, ci, co):
    """Numpy restatement of FEMM's native air-gap element matrix (BuildNativeFemmAirGapMatrix,
    native_airgap_matrix.cpp:5-22, its expanded polynomials from fkn/prob1big.cpp:158-213)
    as T^T Q T: corner values by Catmull-Rom interpolation of four ring nodes at t = 1 - c,
    Q the four-corner form K (5a^2 + 2ab + 5b^2)/12 + Ki (5a'^2 + 2a'b' + 5b'^2)/12."""
    def cr(t):
        return np.array([0.5 * (-t ** 3 + 2 * t ** 2 - t), 0.5 * (3 * t ** 3 - 5 * t ** 2 + 2),
                         0.5 * (-3 * t ** 3 + 4 * t ** 2 + t), 0.5 * (t ** 3 - t ** 2)])
    T = np.zeros((4, 10))
    wi, wo = cr(1.0 - ci), cr(1.0 - co)
    T[0, 0:4], T[1, 1:5], T[2, 5:9], T[3, 6:10] = wi, wi, wo, wo
    d, al, ac, dg = 5 * (K + Ki), Ki - 5 * K, K - 5 * Ki, -(K + Ki)
    Q = np.array([[d, al, ac, dg], [al, d, dg, ac], [ac, dg, d, al], [dg, ac, al, d]]) / 12.0
    return T.T @ Q @ T


def ref_age_matrix(K, Ki, ci, co):
    """The reference's BuildNativeFemmAirGapMatrix (oracle/_ref), or None if it refuses."""
    out = np.zeros(100)
    if ref().ref_age_matrix(C.c_double(K), C.c_double(Ki), C.c_double(ci), C.c_double(co), _p(out)):
        return None
    return out.reshape(10, 10)


def ref_prepared_age(model):
    """PreparedNonlinearAssembly's (status, age_values [nnz], age_rhs [rows]) of a model."""
    r = ref()
    view = ModelView(model)
    h = C.c_void_p()
    st = r.ref_prepare(view.ref(), C.byref(h))
    if st:
        return st, None, None
    vals, rhs = np.zeros(r.ref_prepared_nnz(h)), np.zeros(r.ref_prepared_rows(h))
    r.ref_prepared_age(h, _p(vals), _p(rhs))
    r.ref_prepared_free(h)
    return 0, vals, rhs


def ref_sliding_band_pose(handle, angle_deg):
    """ApplySlidingBandAngle (io/sample_request.cpp:448-491): a new handle posed at angle_deg."""
    r = ref()
    h = C.c_void_p()
    rc = r.ref_sliding_band_pose(handle.h, C.c_double(angle_deg), C.byref(h))
    out = RefHandle(h)
    if rc:
        raise RuntimeError("ApplySlidingBandAngle refused")
    return out


def ref_age_records(handle):
    """The air-gap elements of a handle: [(meta [8], nodes [P, 4], weights [P, 4])], meta =
    antiperiodic, cx, cy, ri, ro, arc degrees, inner shift, outer shift."""
    r = ref()
    out = []
    for b in range(r.ref_age_count(handle.h)):
        P = r.ref_age_points(handle.h, C.c_int32(b))
        meta, nodes, weights = np.zeros(8), np.zeros((P, 4), np.int32), np.zeros((P, 4))
        r.ref_age_copy(handle.h, C.c_int32(b), _p(meta), _p(nodes), _p(weights))
        out.append((meta, nodes, weights))
    return out


def ref_age_postprocess(handle, a, angles_rad=()):
    """ComputeAirGapElementPostprocess: (status, Fx, Fy, torque, radial [angles])."""
    a = np.ascontiguousarray(a, np.float64)
    ang = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
    out3, radial = np.zeros(3), np.zeros(max(ang.size, 1))
    st = ref().ref_age_postprocess(handle.h, _p(a), C.c_int32(ang.size), _p(ang), _p(out3), _p(radial))
    return int(st), out3[0], out3[1], out3[2], radial[:ang.size]


def ref_age_tangent_postprocess(handle, a, da, angles_rad=()):
    """ComputeAirGapElementTangentPostprocess with the base model as tangent model."""
    a = np.ascontiguousarray(a, np.float64)
    da = np.ascontiguousarray(da, np.float64)
    ang = np.ascontiguousarray(np.asarray(angles_rad, np.float64).ravel())
    out3, radial = np.zeros(3), np.zeros(max(ang.size, 1))
    st = ref().ref_age_tangent_postprocess(handle.h, _p(a), _p(da), C.c_int32(ang.size), _p(ang), _p(out3),
                                           _p(radial))
    return int(st), out3[0], out3[1], out3[2], radial[:ang.size]


def ref_artifact_cpu_solve(handle, currents, node_count, circuit_count, options=None, threads=1):
    """The reference CPU Newton path on a handle's model: (a [k, N], flux [k, C], status [k],
    Newton iterations [k])."""
    currents = np.ascontiguousarray(np.atleast_2d(currents), np.float64)
    k = currents.shape[0]
    a, flux = np.zeros((k, node_count)), np.zeros((k, max(circuit_count, 1)))
    status, newton = np.zeros(k, np.int32), np.zeros(k, np.int32)
    opts = options if options is not None else production_options()
    rc = ref().ref_artifact_cpu_solve(handle.h, C.c_int32(k), _p(currents), C.byref(opts), C.c_int32(threads),
                                      _p(a), _p(flux), _p(status), _p(newton))
    if rc:
        raise RuntimeError(f"reference CPU solve status {rc}")
    return a, flux[:, :circuit_count], status, newton
