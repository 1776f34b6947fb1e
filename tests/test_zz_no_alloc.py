"""rf_dense_matvec_noalloc against rf_dense_matvec.

The no-allocation variant exists for callers that cannot let the library
call cudaMalloc (their own pool allocator owns the device memory, or the
allocation latency is not acceptable); it keeps its scratch in a fixed array
in the library's device image instead.  This file is collected last so that a
failure here does not hide the other tests of a run that stops at the first
failure; it also passes when run alone in a fresh process.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _call(fn, A, x, y):
    import torch
    rc = fn(ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
            A.shape[0], ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc


@pytest.mark.parametrize("R", [1500, 4099, 30000])
def test_noalloc_matches_allocating_entry_point_twice(R):
    import torch
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    g = torch.Generator(device="cuda").manual_seed(R)
    # column-major A: column c is A[c*R:(c+1)*R] of the flat buffer
    A = torch.randn(R, R, device="cuda", generator=g)
    for call in range(2):  # the second call must not see the first call's scratch
        x = torch.randn(R, device="cuda", generator=g)
        y_ref = torch.full((R,), float("nan"), device="cuda")
        y_na = torch.full((R,), float("nan"), device="cuda")
        assert _call(lib.rf_dense_matvec, A, x, y_ref) == C.RF_OK
        assert _call(lib.rf_dense_matvec_noalloc, A, x, y_na) == C.RF_OK, lib.rf_last_error()
        tol = 1e-4 * float(A.abs().max()) * R ** 0.5
        assert torch.isfinite(y_na).all()
        assert torch.allclose(y_na, y_ref, rtol=1e-4, atol=tol), (call, float((y_na - y_ref).abs().max()))
        exact = (A.t().double() @ x.double()).float()  # A stored column-major = A.t() row-major
        assert torch.allclose(y_na, exact, rtol=1e-4, atol=tol)


def test_noalloc_rejects_rows_beyond_its_scratch():
    import torch
    from rigidfibers_b200 import _capi as C
    lib = C.load()
    dummy = torch.zeros(4, device="cuda")
    rc = lib.rf_dense_matvec_noalloc(ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()),
                                     ctypes.c_void_p(dummy.data_ptr()), 131073, None)
    assert rc == C.RF_E_INPUT
    assert b"131072" in lib.rf_last_error()
