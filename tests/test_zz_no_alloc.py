"""fg_csr_pcg_noalloc: the PCG for callers that may not allocate GPU memory.

Such callers -- code inside a memory pool that owns the device, real-time loops that
forbid allocator calls, plug-in hosts that lend only their own buffers -- hand the
library a CSR system and a solution buffer in device memory they already own, and the
library works out of one fixed device array instead of allocating.  Through the C ABI
this checks that:
* two calls in a row give the same answers as the allocating entry point fg_csr_pcg
  (same statuses and iteration counts, solutions within 1e-12 relative) and as the CPU
  oracle's PCG (the 3x3 system's exact answer to 1e-13; the assembled system within
  1e-6 relative, the bound the PCG parity tests use at tolerance 1e-10);
* after the first call (which loads the library's device code and its array) further
  calls change the device's free memory by nothing (cudaMemGetInfo);
* a bad tolerance or iteration budget returns FG_OK with INVALID_ARGUMENT in info, as the
  allocating entry does; bad offsets, out-of-range columns and non-finite values are
  refused with FG_INVALID_ARGUMENT; systems beyond the stated limits are refused;
* a valid call after refused ones still answers correctly (the shared array is rewritten).
The file is named to be collected last so a run that stops at the first failure has run
every other test already.
"""
import numpy as np
import pytest

import femm_gpu_b200 as fg
import oracle as O
from femm_gpu_b200 import meshes

pytestmark = pytest.mark.gpu


def device(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def systems():
    # The reference's 3x3 known answer (self_test.cu:33-53) and an assembled Newton system.
    yield (np.array([0, 2, 5, 7], np.int32), np.array([0, 1, 0, 1, 2, 1, 2], np.int32),
           np.array([4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 3.0]), np.array([4.0, 4.0, 3.0]),
           np.array([2.0, 4.0, 7.0]), 1e-13)
    model = meshes.square_nonlinear(m=40, seed=12)
    rng = np.random.default_rng(4)
    a = rng.normal(size=model.node_count) * 1e-3
    a[model.dir_nodes] = 0.0
    s = O.assemble(model, a, [3.0, -5.0, 8.0], 1)
    yield s.off, s.col, s.val, s.diag, s.rhs, 1e-10


@pytest.mark.parametrize("idx", [0, 1])
def test_noalloc_matches_allocating_entry_on_two_calls(gpu, idx):
    import torch

    ro, col, val, diag, rhs, tol = list(systems())[idx]
    n = ro.size - 1
    x_ref, info_ref = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=tol, maxit=16384)
    bufs = [device(ro, torch), device(col, torch), device(val, torch), device(diag, torch),
            device(rhs, torch)]
    for call in range(2):
        x = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        status, info = fg.capi.csr_pcg_noalloc(n, *[b.data_ptr() for b in bufs], x.data_ptr(),
                                               tol=tol, maxit=16384)
        assert status == fg.capi.OK, (call, status)
        assert info.status == info_ref[0].status == fg.capi.OK
        assert info.iterations == info_ref[0].iterations
        got = x.cpu().numpy()
        assert np.linalg.norm(got - x_ref[0]) <= 1e-12 * np.linalg.norm(x_ref[0]), call
    st, x_or, _, _ = O.pcg(O.csr_system(ro, col, val, rhs), tol=tol, maxit=16384)
    assert st == 0
    bound = 1e-13 if idx == 0 else 1e-6
    assert np.linalg.norm(got - x_or) <= bound * np.linalg.norm(x_or)


def test_noalloc_allocates_nothing_after_the_first_call(gpu):
    import torch

    ro, col, val, diag, rhs, tol = list(systems())[1]
    n = ro.size - 1
    bufs = [device(ro, torch), device(col, torch), device(val, torch), device(diag, torch),
            device(rhs, torch)]
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    ptrs = [b.data_ptr() for b in bufs] + [x.data_ptr()]
    status, _ = fg.capi.csr_pcg_noalloc(n, *ptrs, tol=tol)
    assert status == fg.capi.OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        status, info = fg.capi.csr_pcg_noalloc(n, *ptrs, tol=tol)
        assert status == fg.capi.OK and info.status == fg.capi.OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_status_cases_and_refusals(gpu):
    import torch

    ro, col, val, diag, rhs, _ = next(iter(systems()))
    bufs = [device(ro, torch), device(col, torch), device(val, torch), device(diag, torch),
            device(rhs, torch)]
    x = torch.zeros(3, dtype=torch.float64, device="cuda")
    ptrs = [b.data_ptr() for b in bufs] + [x.data_ptr()]
    # A bad tolerance or budget: the call succeeds and the solve reports INVALID_ARGUMENT
    # (GpuCsrSolver::Solve's argument rule), as fg_csr_pcg does.
    for tol, maxit in ((0.0, 64), (-1e-10, 64), (1.0, 64), (float("nan"), 64), (1e-10, -1)):
        status, info = fg.capi.csr_pcg_noalloc(3, *ptrs, tol=tol, maxit=maxit)
        assert status == fg.capi.OK and info.status == fg.capi.INVALID_ARGUMENT, (tol, maxit)
        _, ref = fg.csr_pcg(ro, col, val, diag, rhs[None, :], tol=tol, maxit=maxit)
        assert ref[0].status == fg.capi.INVALID_ARGUMENT
    # Refused systems: offsets not starting at 0, a column outside [0, n), a NaN value.
    bad_ro = device(np.array([1, 3, 6, 7], np.int32), torch)
    bad_col = device(np.array([0, 1, 0, 1, 3, 1, 2], np.int32), torch)
    bad_val = device(np.array([4.0, -1.0, -1.0, np.nan, -1.0, -1.0, 3.0]), torch)
    for i, bad in ((0, bad_ro), (1, bad_col), (2, bad_val)):
        args = list(ptrs)
        args[i] = bad.data_ptr()
        status, info = fg.capi.csr_pcg_noalloc(3, *args, tol=1e-13)
        assert status == fg.capi.INVALID_ARGUMENT and info.status == fg.capi.INVALID_ARGUMENT, i
    status, info = fg.capi.csr_pcg_noalloc(3, *ptrs, tol=1e-13)
    assert status == fg.capi.OK and info.status == fg.capi.OK
    np.testing.assert_allclose(x.cpu().numpy(), [1.0, 2.0, 3.0], rtol=1e-13)


def test_noalloc_refuses_systems_beyond_its_limits(gpu):
    import torch

    n = fg.capi.NOALLOC_MAX_ROWS + 1
    ro = device(np.arange(n + 1, dtype=np.int32), torch)
    col = device(np.arange(n, dtype=np.int32), torch)
    ones = device(np.ones(n), torch)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    status, info = fg.capi.csr_pcg_noalloc(n, ro.data_ptr(), col.data_ptr(), ones.data_ptr(),
                                           ones.data_ptr(), ones.data_ptr(), x.data_ptr())
    assert status == fg.capi.INVALID_ARGUMENT
    # Within the row limit but beyond the slot limit: one dense row widens its slice.
    n = 8192
    lens = np.ones(n, np.int64)
    lens[0] = n  # slice 0 padded to width n: 32 * 8192 slots > FG_NOALLOC_MAX_POSITIONS
    ro_np = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col_np = np.concatenate([np.arange(n), np.arange(1, n)]).astype(np.int32)
    val_np = np.ones(col_np.size)
    bufs = [device(ro_np, torch), device(col_np, torch), device(val_np, torch),
            device(np.ones(n), torch), device(np.ones(n), torch)]
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    status, info = fg.capi.csr_pcg_noalloc(n, *[b.data_ptr() for b in bufs], x.data_ptr())
    assert status == fg.capi.INVALID_ARGUMENT
    # ... and a valid call afterwards still answers correctly (the shared array is rewritten).
    ro, col, val, diag, rhs, tol = next(iter(systems()))
    bufs = [device(ro, torch), device(col, torch), device(val, torch), device(diag, torch),
            device(rhs, torch)]
    x = torch.zeros(3, dtype=torch.float64, device="cuda")
    status, info = fg.capi.csr_pcg_noalloc(3, *[b.data_ptr() for b in bufs], x.data_ptr(), tol=tol)
    assert status == fg.capi.OK and info.status == fg.capi.OK
    np.testing.assert_allclose(x.cpu().numpy(), [1.0, 2.0, 3.0], rtol=1e-13)
