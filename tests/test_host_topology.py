"""Host-side logic, no GPU: the library's plan topology against the reference.

* symbolic CSR, free-row numbering and signed node maps must be bit-exact
  (gpu_solver/src/physics/nonlinear_topology.cpp:12-137, signed_node_constraints.h:33-106);
  -- on small meshes and on the benchmark's full-size workloads;
* the per-slot / per-row contributor lists and the fixed PM / coil loads must equal the
  reference's PreparedNonlinearAssembly (nonlinear_topology.cpp:87-248);
* the oracle's host assembler must reproduce the reference's AssembleNonlinearNewton
  bit for bit (nonlinear_model.cpp:453-627).
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes

REF = O.ref()
needs_ref = pytest.mark.skipif(REF is None, reason="oracle/_ref not built (no reference checkout)")

PAIR = np.array([[0, 1, 2], [1, 3, 4], [2, 4, 5]])


def models():
    yield meshes.square_nonlinear(m=12, seed=5)
    yield meshes.square_linear(m=10)
    yield meshes.periodic_strip(m=8)
    yield meshes.periodic_strip(m=8, antiperiodic=True)
    yield meshes.axisymmetric_plunger(mr=8, mz=12)


# The workloads the benchmark measures, built when their test runs: the 251,001-node
# nonlinear planar square (m = 500, seed 2), the 40,411-node anti-periodic rotor-stator
# sector and the 2,002,225-node planar square (m = 1414).
HEADLINE = {"square_nonlinear_m500": lambda: meshes.square_nonlinear(m=500, seed=2),
            "annular_sector": lambda: meshes.annular_sector(),
            "square_nonlinear_m1414": lambda: meshes.square_nonlinear(m=1414, seed=2)}


def cases(include_headline):
    out = [pytest.param(m, id=m.name) for m in models()]
    return out + [pytest.param(name, id=name) for name in include_headline]


def as_model(model):
    return HEADLINE[model]() if isinstance(model, str) else model


def ref_prepared(model):
    import ctypes as C
    view = O.ModelView(model)
    h = C.c_void_p()
    assert REF.ref_prepare(view.ref(), C.byref(h)) == 0
    rows, nnz = REF.ref_prepared_rows(h), REF.ref_prepared_nnz(h)
    me, re = REF.ref_prepared_matrix_entries(h), REF.ref_prepared_rhs_entries(h)
    out = dict(ro=np.zeros(rows + 1, np.int32), col=np.zeros(nnz, np.int32),
               free=np.zeros(rows, np.int32), moff=np.zeros(nnz + 1, np.int32),
               ment=np.zeros(4 * me, np.int32), roff=np.zeros(rows + 1, np.int32),
               rent=np.zeros(3 * re, np.int32), pm=np.zeros(rows),
               cr=np.zeros(max(model.circuit_count, 1) * rows), dslot=np.zeros(rows, np.int32))
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    REF.ref_prepared_copy(h, p(out["ro"]), p(out["col"]), p(out["free"]), p(out["moff"]),
                          p(out["ment"]), p(out["roff"]), p(out["rent"]), p(out["pm"]), p(out["cr"]),
                          p(out["dslot"]))
    REF.ref_prepared_free(h)
    out["ment"] = out["ment"].reshape(-1, 4)
    out["rent"] = out["rent"].reshape(-1, 3)
    return out


@needs_ref
@pytest.mark.parametrize("model", cases(list(HEADLINE)))
def test_symbolic_csr_and_maps_bit_exact(model):
    model = as_model(model)
    plan = fg.Plan(model, host_only=True)
    ro, col, n2f, sign, bnd = plan.symbolic()
    ref = ref_prepared(model)
    assert np.array_equal(ro, ref["ro"])
    assert np.array_equal(col, ref["col"])
    rc, root, rsign, rn2f, rbnd, nf = O.signed_dofs(model.node_count, model.con_a, model.con_b,
                                                    model.con_sign, model.dir_nodes, model.dir_values)
    assert rc == 0 and nf == plan.rows
    assert np.array_equal(n2f, rn2f) and np.array_equal(sign, rsign)
    assert np.array_equal(bnd, rbnd)
    # free rows are numbered by ascending root node
    free_roots = np.flatnonzero((root == np.arange(model.node_count)) & (n2f >= 0))
    assert np.array_equal(free_roots, ref["free"])


@needs_ref
@pytest.mark.parametrize("model", cases(["square_nonlinear_m500", "annular_sector"]))
def test_contributors_and_fixed_loads_match_reference(model):
    model = as_model(model)
    plan = fg.Plan(model, host_only=True)
    so, se, ro, re, pm, cr = plan.contributors()
    ref = ref_prepared(model)
    assert np.array_equal(so, ref["moff"])
    m = ref["ment"]
    assert np.array_equal(se[:, 0], m[:, 0])
    assert np.array_equal(se[:, 1], PAIR[m[:, 1], m[:, 2]])
    assert np.array_equal(se[:, 2], m[:, 3])
    assert np.array_equal(ro, ref["roff"])
    assert np.array_equal(re, ref["rent"])
    assert np.array_equal(pm, ref["pm"])
    assert np.array_equal(cr.ravel(), ref["cr"][: cr.size])


@needs_ref
@pytest.mark.parametrize("model", list(models()), ids=lambda m: m.name)
@pytest.mark.parametrize("use_newton", [0, 1])
def test_oracle_assembler_is_the_reference(model, use_newton):
    rng = np.random.default_rng(7)
    a = rng.normal(size=model.node_count) * 2e-3
    cur = rng.uniform(-10, 10, size=model.circuit_count)
    mine = O.assemble(model, a, cur, use_newton)
    theirs = O.assemble(model, a, cur, use_newton, use_ref=True)
    assert np.array_equal(mine.off, theirs.off) and np.array_equal(mine.col, theirs.col)
    assert np.array_equal(mine.val, theirs.val)
    assert np.array_equal(mine.rhs, theirs.rhs)
    assert np.array_equal(mine.diag, theirs.diag)


@needs_ref
def test_oracle_validation_statuses_match_reference():
    base = meshes.square_nonlinear(m=6, seed=1)
    cases = []
    m = meshes.square_nonlinear(m=6, seed=1)
    m.tri = m.tri[:, [0, 2, 1]].copy()  # clockwise
    cases.append(m)
    m = meshes.square_nonlinear(m=6, seed=1)
    m.tri_mat = m.tri_mat.copy()
    m.tri_mat[0] = 99
    cases.append(m)
    m = meshes.square_nonlinear(m=6, seed=1)
    m.dir_nodes = np.concatenate([m.dir_nodes, m.dir_nodes[:1]]).astype(np.int32)
    m.dir_values = np.zeros(m.dir_nodes.size)
    cases.append(m)
    m = meshes.square_nonlinear(m=6, seed=1)
    m.circuit_index = m.circuit_index.copy()
    m.circuit_index[3] = 7
    cases.append(m)
    for case in [base] + cases:
        assert O.validate(case) == O.validate(case, use_ref=True)
    assert O.validate(base) == 0
    assert [O.validate(c) for c in cases] == [4, 15, 5, 15]
    # the library's host-only plan reports the same statuses
    for case in cases:
        with pytest.raises(fg.FgError) as err:
            fg.Plan(case, host_only=True)
        assert err.value.status == O.validate(case)


def test_signed_dof_contradictions():
    # A(1) = A(0), A(2) = -A(1), A(0) = A(2) -> contradictory cycle (status 2)
    rc = O.signed_dofs(4, [0, 1, 2], [1, 2, 0], np.array([1, -1, 1], np.int8), [3], [0.0])[0]
    assert rc == 2
    # self-pair anti-periodic is contradictory, periodic self-pair is invalid
    assert O.signed_dofs(3, [1], [1], np.array([-1], np.int8), [0], [0.0])[0] == 2
    assert O.signed_dofs(3, [1], [1], np.array([1], np.int8), [0], [0.0])[0] == 1
    if REF is not None:
        import ctypes as C
        for (a, b, s) in (([0, 1, 2], [1, 2, 0], [1, -1, 1]),):
            arrs = [np.array(a, np.int32), np.array(b, np.int32), np.array(s, np.int8)]
            root = np.zeros(4, np.int32)
            sign = np.zeros(4, np.int8)
            r2f = np.zeros(4, np.int32)
            nf = C.c_int32()
            p = lambda x: x.ctypes.data_as(C.c_void_p)  # noqa: E731
            rc = REF.ref_signed_dofs(4, 3, p(arrs[0]), p(arrs[1]), p(arrs[2]), 1,
                                     p(np.array([3], np.int32)), p(np.array([0.0])), p(root),
                                     p(sign), p(r2f), C.byref(nf))
            assert rc == 2


def test_library_exports_every_header_symbol():
    import ctypes as C
    import os
    import re
    header = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "femm_gpu.h")).read()
    declared = set(re.findall(r"\b(fg_[a-z_]+)\s*\(", header))
    lib = C.CDLL(fg.LIB_PATH)
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing, missing
    assert set(fg.EXPORTED) <= declared
    assert fg.lib().fg_abi_version() == 2
    assert fg.status_name(14) == "NONLINEAR_SOLVE_NOT_CONVERGED"


def test_device_calls_refuse_without_gpu_on_host_only_plan():
    plan = fg.Plan(meshes.square_linear(m=6), host_only=True)
    with pytest.raises(fg.FgError) as err:
        plan.solve([[10.0]])
    assert err.value.status == fg.capi.GPU_UNAVAILABLE


def test_preconditioner_options_are_validated():
    model = meshes.square_linear(m=6)
    for bs in (8, 32):
        fg.Plan(model, preconditioner=1, block_size=bs, host_only=True)
        fg.Plan(model, preconditioner=1, block_size=bs, precision=1, host_only=True)
    for pre, bs in ((1, 16), (1, 0), (2, 8)):
        with pytest.raises(fg.FgError) as e:
            fg.Plan(model, preconditioner=pre, block_size=bs, host_only=True)
        assert e.value.status == fg.capi.UNSUPPORTED_FEATURE


def test_one_reduction_form_is_fp64_jacobi_only():
    """FG_PLAN_PCG_ONE_REDUCTION exists for the FP64 Jacobi method alone."""
    model = meshes.square_linear(m=6)
    fg.Plan(model, one_reduction=True, host_only=True)
    fg.Plan(model, one_reduction=True, from_iterate=True, host_only=True)
    for form in (dict(precision=1), dict(preconditioner=1, block_size=8)):
        with pytest.raises(fg.FgError) as e:
            fg.Plan(model, one_reduction=True, host_only=True, **form)
        assert e.value.status == fg.capi.UNSUPPORTED_FEATURE
