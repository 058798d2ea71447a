"""The allocation-free entry point splab_gemm_dmma_noalloc (include/splab.h),
for callers that cannot allocate device memory, against the existing entry
point splab_gemm on the same inputs: same result within the FP64 tolerance of
the other tests, on two calls in a row (the static scratch array keeps the
previous call's contents), and its size limit. Collected last on purpose."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    import spla_b200
    L = spla_b200.lib()
    vp, i, i64 = ct.c_void_p, ct.c_int, ct.c_int64
    L.splab_gemm_dmma_noalloc.argtypes = [i, i, i, i64, i64, i64, vp, vp, i64, vp, i64, vp, vp,
                                          i64, i, i64, i64, vp]
    L.splab_gemm_dmma_noalloc.restype = i
    return spla_b200, L


def _rel(x, y):
    return float(np.linalg.norm((x - y).ravel()) / np.linalg.norm(y.ravel()))


@pytest.mark.parametrize("dtype,opA,m,n,k", [("complex128", 2, 300, 200, 60000),
                                             ("float64", 1, 257, 129, 40000),
                                             ("complex128", 0, 96, 80, 5000)])
def test_noalloc_matches_splab_gemm_twice(dtype, opA, m, n, k):
    import torch
    spla, L = _lib()
    tdt = getattr(torch, dtype)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    # op(A) is m x k: A stored k x m for T/C, m x k for N
    lda = k if opA else m
    A = torch.randn(lda * (m if opA else k), dtype=tdt, device="cuda", generator=g)
    B = torch.randn(k * n, dtype=tdt, device="cuda", generator=g)
    C0 = torch.randn(m * n, dtype=tdt, device="cuda", generator=g)
    alpha = (ct.c_double * 2)(0.75, -0.25)
    beta = (ct.c_double * 2)(0.5, 0.125)
    # existing entry point, with its own workspace
    ws_bytes = spla.splab_gemm_workspace_size(dtype, 1, opA, 0, m, n, k)
    ws = torch.empty(max(1, ws_bytes), dtype=torch.uint8, device="cuda")
    C_ref = C0.clone()
    rc = spla.lib().splab_gemm(spla._dtype_of(dtype=dtype), 1, opA, 0, m, n, k,
                               ct.cast(alpha, ct.c_void_p), A.data_ptr(), lda, B.data_ptr(), k,
                               ct.cast(beta, ct.c_void_p), C_ref.data_ptr(), m, 0, 0, 0, 0,
                               ws.data_ptr(), ws_bytes, 0)
    assert rc == 0
    torch.cuda.synchronize()
    ref = C_ref.cpu().numpy()
    for call in range(2):
        C = C0.clone()
        rc = L.splab_gemm_dmma_noalloc(spla._dtype_of(dtype=dtype), opA, 0, m, n, k,
                                       ct.cast(alpha, ct.c_void_p), A.data_ptr(), lda,
                                       B.data_ptr(), k, ct.cast(beta, ct.c_void_p), C.data_ptr(),
                                       m, 0, 0, 0, 0)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        err = _rel(C.cpu().numpy(), ref)
        assert err <= 1e-14, (call, err)


def test_noalloc_rejects_problems_beyond_the_static_scratch():
    import torch
    spla, L = _lib()
    m = n = 2048  # complex: m * n * 16 = 64 MiB > 32 MiB
    k = 64
    A = torch.zeros(k * m, dtype=torch.complex128, device="cuda")
    B = torch.zeros(k * n, dtype=torch.complex128, device="cuda")
    C = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    one = (ct.c_double * 2)(1.0, 0.0)
    zero = (ct.c_double * 2)(0.0, 0.0)
    rc = L.splab_gemm_dmma_noalloc(3, 2, 0, m, n, k, ct.cast(one, ct.c_void_p), A.data_ptr(), k,
                                   B.data_ptr(), k, ct.cast(zero, ct.c_void_p), C.data_ptr(), m,
                                   0, 0, 0, 0)
    assert rc == 2  # SPLAB_ERR_WORKSPACE
