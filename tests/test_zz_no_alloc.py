"""The allocation-free entry point splab_gemm_dmma_noalloc (include/splab.h),
for callers that cannot allocate device memory (a framework allocator that
owns every byte, a hard device-memory cap, loops that cannot take the
synchronisation of cudaMalloc / cudaFree). Checked against the existing entry
point splab_gemm on the same inputs and against the double-double oracle, on
two calls in a row (the static scratch array keeps the previous call's
contents), on each of its branches: the planner's own split count, fewer
splits so that the partials fit the static array, no partials at all (one
split) for a C larger than the array, and the refusal of a problem whose
partials cannot fit. Collected last on purpose."""
import ctypes as ct

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SCRATCH = 64 << 20  # SPLAB_NOALLOC_SCRATCH_BYTES


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


def _noalloc(L, code, opA, m, n, k, scalars, A, lda, B, C):
    """One call through the C ABI; scalars = (alpha, beta) as ctypes double pairs."""
    a, b = [ct.cast(v, ct.c_void_p) for v in scalars]
    return L.splab_gemm_dmma_noalloc(code, opA, 0, m, n, k, a, A.data_ptr(), lda, B.data_ptr(), k,
                                     b, C.data_ptr(), m, 0, 0, 0, 0)


def _oracle(dtype, opA, m, n, k, A, lda, B, C0, cols, alpha, beta):
    """alpha op(A) B + beta C0 on columns `cols`, CPU double-double."""
    An = A.cpu().numpy()
    Bn = np.ascontiguousarray(B.view(n, k)[cols].cpu().numpy().ravel())
    ref = np.ascontiguousarray(C0.view(n, m)[cols].cpu().numpy().ravel())
    assert oracle.gemm(opA, 0, m, len(cols), k, alpha, An, lda, Bn, k, beta, ref, m) == 0
    return ref


CASES = [  # dtype, opA, m, n, k, which branch
    ("complex128", 2, 300, 200, 60000, "planner splits"),
    ("float64", 1, 257, 129, 40000, "planner splits"),
    ("complex128", 0, 96, 80, 5000, "planner splits"),
    ("complex128", 2, 1024, 1024, 200000, "fewer splits"),
    ("complex128", 2, 2048, 2048, 64, "one split, C larger than the array"),
]


@pytest.mark.parametrize("dtype,opA,m,n,k,branch", CASES, ids=[c[5] + f" {c[2]}x{c[3]}x{c[4]}"
                                                               for c in CASES])
def test_noalloc_matches_splab_gemm_and_oracle_twice(dtype, opA, m, n, k, branch):
    import torch
    spla, L = _lib()
    code = spla._dtype_of(dtype=dtype)
    esz = 16 if "complex" in dtype else 8
    ws_bytes = spla.splab_gemm_workspace_size(dtype, 1, opA, 0, m, n, k)
    # the case exercises the branch it is named for
    if branch == "fewer splits":
        assert ws_bytes > SCRATCH and 2 * m * n * esz <= SCRATCH, ws_bytes
    elif branch.startswith("one split"):
        assert ws_bytes == 0 and 2 * m * n * esz > SCRATCH, ws_bytes
    else:
        assert 0 < ws_bytes <= SCRATCH, ws_bytes
    tdt = getattr(torch, dtype)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    # op(A) is m x k: A stored k x m for T/C, m x k for N
    lda = k if opA else m
    s = (1.0 / k) ** 0.5
    A = torch.randn(lda * (m if opA else k), dtype=tdt, device="cuda", generator=g) * s
    B = torch.randn(k * n, dtype=tdt, device="cuda", generator=g) * s
    C0 = torch.randn(m * n, dtype=tdt, device="cuda", generator=g)
    av, bv = complex(0.75, -0.25), complex(0.5, 0.125)
    if "complex" not in dtype:
        av, bv = av.real, bv.real
    alpha = (ct.c_double * 2)(complex(av).real, complex(av).imag)
    beta = (ct.c_double * 2)(complex(bv).real, complex(bv).imag)
    # existing entry point, with its own workspace
    ws = torch.empty(max(1, ws_bytes), dtype=torch.uint8, device="cuda")
    C_ref = C0.clone()
    rc = spla.lib().splab_gemm(code, 1, opA, 0, m, n, k, ct.cast(alpha, ct.c_void_p),
                               A.data_ptr(), lda, B.data_ptr(), k, ct.cast(beta, ct.c_void_p),
                               C_ref.data_ptr(), m, 0, 0, 0, 0, ws.data_ptr(), ws_bytes, 0)
    assert rc == 0
    torch.cuda.synchronize()
    del ws
    ref = C_ref.cpu().numpy()
    cols = [0, n // 2, n - 1]
    dd = _oracle(dtype, opA, m, n, k, A, lda, B, C0, cols, av, bv)
    for call in range(2):
        C = C0.clone()
        assert _noalloc(L, code, opA, m, n, k, (alpha, beta), A, lda, B, C) == 0, call
        torch.cuda.synchronize()
        got = C.cpu().numpy()
        assert _rel(got, ref) <= 1e-14, (call, _rel(got, ref))
        err = oracle.rel_fro(got.reshape(n, m)[cols].ravel(), dd)
        assert err <= 1e-14, (call, err)


def test_noalloc_rejects_partials_beyond_the_static_scratch():
    """A problem that the planner splits along k, with C too large for two
    FP64 partials (complex 2048 x 2048: 64 MiB each), is refused with
    SPLAB_ERR_WORKSPACE and leaves C unchanged."""
    import torch
    spla, L = _lib()
    m = n = 2048
    k = 100000
    assert spla.splab_gemm_workspace_size("complex128", 1, 2, 0, m, n, k) > 0  # split along k
    A = torch.zeros(k * m, dtype=torch.complex128, device="cuda")
    B = torch.zeros(k * n, dtype=torch.complex128, device="cuda")
    C = torch.full((m * n,), 3.0 + 1.0j, dtype=torch.complex128, device="cuda")
    one = (ct.c_double * 2)(1.0, 0.0)
    zero = (ct.c_double * 2)(0.0, 0.0)
    assert _noalloc(L, 3, 2, m, n, k, (one, zero), A, k, B, C) == 2  # SPLAB_ERR_WORKSPACE
    torch.cuda.synchronize()
    assert bool(torch.all(C == 3.0 + 1.0j))
