"""The no-allocation entry point, nir_pdhg_reference_solve_noalloc.

It serves callers that cannot call cudaMalloc (their device memory belongs
to their own pool allocator, or they may not take cudaMalloc's implicit
device synchronisation): the caller hands over an LP already resident in
device memory, and the entry point runs the reference PDHG loop using only
a fixed file-scope device array as scratch.  This test is the caller: it
places the LP in device memory with torch, calls the entry point through
the C ABI twice in a row, and requires the result of each call to equal,
bit for bit, what the allocating entry point (nir_pdhg_solve with
NIR_ALGO_REFERENCE) returns for the same LP.  It also checks that an LP
beyond the scratch limit is rejected with a clear error.

Kept in its own file, collected last, so that a failure here never hides
the other tests of a run that stops at the first failure.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu
from nirnaya_b200 import lp as L
from nirnaya_b200 import pdhg

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")]


class CsrDev(C.Structure):
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p),
                ("value", C.c_void_p)]


def _bind():
    lib = pdhg.lib()
    fn = lib.nir_pdhg_reference_solve_noalloc
    D = C.c_void_p
    fn.argtypes = [C.POINTER(CsrDev), C.POINTER(CsrDev), D, D, D, D, D, C.c_int64, C.c_void_p, D, D,
                   C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    fn.restype = C.c_int
    return fn


def _device_lp(lp, torch):
    """CSR of A and of A' (the CSC of A) as device tensors."""
    dev = "cuda:0"
    cols = np.repeat(np.arange(lp.ncol, dtype=np.int32), np.diff(lp.col_start))
    order = np.argsort(lp.row_index, kind="stable")  # each row keeps ascending columns
    a_ci = cols[order]
    a_val = lp.value[order]
    a_rp = np.concatenate([[0], np.cumsum(np.bincount(lp.row_index, minlength=lp.nrow))]).astype(np.int32)
    t = {
        "a_rp": torch.tensor(a_rp, dtype=torch.int32, device=dev),
        "a_ci": torch.tensor(a_ci, dtype=torch.int32, device=dev),
        "a_val": torch.tensor(a_val, dtype=torch.float64, device=dev),
        "t_rp": torch.tensor(lp.col_start.astype(np.int32), dtype=torch.int32, device=dev),
        "t_ci": torch.tensor(lp.row_index, dtype=torch.int32, device=dev),
        "t_val": torch.tensor(lp.value, dtype=torch.float64, device=dev),
    }
    for k in ("cost", "collo", "colup", "rowlo", "rowup"):
        t[k] = torch.tensor(getattr(lp, k), dtype=torch.float64, device=dev)
    A = CsrDev(lp.nrow, lp.ncol, t["a_rp"].data_ptr(), t["a_ci"].data_ptr(), t["a_val"].data_ptr())
    At = CsrDev(lp.ncol, lp.nrow, t["t_rp"].data_ptr(), t["t_ci"].data_ptr(), t["t_val"].data_ptr())
    return A, At, t


def _call(fn, A, At, t, max_iters, torch, lp):
    x = torch.zeros(lp.ncol, dtype=torch.float64, device="cuda:0")
    y = torch.zeros(lp.nrow, dtype=torch.float64, device="cuda:0")
    it = C.c_int64(-1)
    st = C.c_int32(-1)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(C.byref(A), C.byref(At), t["cost"].data_ptr(), t["collo"].data_ptr(), t["colup"].data_ptr(),
            t["rowlo"].data_ptr(), t["rowup"].data_ptr(), max_iters, stream, x.data_ptr(), y.data_ptr(),
            C.byref(it), C.byref(st))
    torch.cuda.synchronize()
    return rc, x.cpu().numpy(), y.cpu().numpy(), it.value, st.value


@pytest.mark.parametrize("kind,kw,max_iters", [
    (L.RANDOM_EQ, dict(m=300, n=700), 4000),
    (L.MULTIPERIOD, dict(m=480), 3000),
])
def test_noalloc_matches_allocating_entry_point_twice(kind, kw, max_iters):
    torch = pytest.importorskip("torch")
    fn = _bind()
    lp = L.generate(kind, 13, **kw)
    with pdhg.Engine(lp) as eng:
        xr, yr, info = eng.solve(pdhg.default_params(algorithm=pdhg.ALGO_REFERENCE, max_iters=max_iters))
    A, At, t = _device_lp(lp, torch)
    for _ in range(2):  # the scratch keeps the previous call's contents
        rc, x, y, it, st = _call(fn, A, At, t, max_iters, torch, lp)
        assert rc == st == info.status, (rc, st, info.status, pdhg.last_error())
        assert it == info.iterations
        # the same kernels in the same order: bit-identical
        assert np.array_equal(x.view(np.int64), xr.view(np.int64))
        assert np.array_equal(y.view(np.int64), yr.view(np.int64))


def test_noalloc_rejects_lp_beyond_scratch_limit():
    torch = pytest.importorskip("torch")
    fn = _bind()
    lp = L.generate(L.RANDOM_EQ, 1, m=20, n=50)
    A, At, t = _device_lp(lp, torch)
    big_A = CsrDev(1 << 20, 50, A.row_ptr, A.col_idx, A.value)
    big_At = CsrDev(50, 1 << 20, At.row_ptr, At.col_idx, At.value)
    x = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    it, st = C.c_int64(0), C.c_int32(0)
    rc = fn(C.byref(big_A), C.byref(big_At), t["cost"].data_ptr(), t["collo"].data_ptr(), t["colup"].data_ptr(),
            t["rowlo"].data_ptr(), t["rowup"].data_ptr(), 10, None, x.data_ptr(), x.data_ptr(), C.byref(it),
            C.byref(st))
    assert rc == pdhg.INPUT_ERROR
    assert "too large" in pdhg.last_error()
