"""The device double-double reference product (splab_gemm_dd) against the CPU
Dot2 oracle: both are compensated dot products, so their double-double
results (hi + lo) agree to about 1e-25 of sum |a||b| (a plain double
product differs at 1e-16), for every dtype
and op pair. This pins the device reference that the full-size accuracy
checks (tests and bench.py) compare against."""
import numpy as np
import pytest

import oracle
from inputs import buffer

pytestmark = pytest.mark.gpu

REAL = {np.float32: np.float64, np.float64: np.float64, np.complex64: np.complex128,
        np.complex128: np.complex128}
CODE = {np.float32: 0, np.float64: 1, np.complex64: 2, np.complex128: 3}


def _abs_product_bound(dt, opA, opB, m, n, k, A, lda, B, ldb):
    """sum_l |op(A)_il| |op(B)_lj| (real-part magnitudes for complex), float64."""
    def mat(X, ld, rows, cols):
        return np.abs(X[: ld * cols].reshape(cols, ld)[:, :rows].T).astype(np.float64)
    a = mat(A, lda, m if opA == 0 else k, k if opA == 0 else m)
    b = mat(B, ldb, k if opB == 0 else n, n if opB == 0 else k)
    a = a if opA == 0 else a.T
    b = b if opB == 0 else b.T
    return a @ b


@pytest.mark.parametrize("dt", [np.float32, np.float64, np.complex64, np.complex128])
@pytest.mark.parametrize("ops", [(0, 0), (1, 0), (2, 0), (0, 1), (2, 2), (1, 2)])
def test_dd_matches_cpu_dot2(spla_lib, dt, ops):
    import torch
    opA, opB = ops
    m, n, k = 37, 29, 1999
    lda = (m if opA == 0 else k) + 3
    ldb = (k if opB == 0 else n) + 2
    A = buffer(dt, lda, k if opA == 0 else m, 101, "gauss_k", k)
    B = buffer(dt, ldb, n if opB == 0 else k, 102, "gauss_k", k)
    rdt = REAL[dt]
    ref = np.zeros(m * n, rdt)
    ref_lo = np.zeros(m * n * (2 if np.iscomplexobj(ref) else 1), np.float64)
    Ad, Bd = A.astype(rdt), B.astype(rdt)  # float inputs: exact in double
    assert oracle.gemm(opA, opB, m, n, k, 1.0, Ad, lda, Bd, ldb, 0.0, ref, m, ref_lo) == 0
    tdt = torch.complex128 if np.iscomplexobj(ref) else torch.float64
    hi = torch.zeros(m * n, dtype=tdt, device="cuda")
    lo = torch.zeros(m * n, dtype=tdt, device="cuda")
    rc = spla_lib.gemm_dd(CODE[dt], opA, opB, m, n, k, torch.from_numpy(A).cuda(), lda,
                          torch.from_numpy(B).cuda(), ldb, hi, m, lo)
    assert rc == 0
    torch.cuda.synchronize()
    gh = hi.cpu().numpy().view(np.float64)
    gl = lo.cpu().numpy().view(np.float64)
    rh = ref.view(np.float64)
    # (hi - hi') is exact for close values; the lo parts carry the rest
    diff = np.abs((gh - rh) + (gl - ref_lo))
    bound = _abs_product_bound(dt, opA, opB, m, n, k, A, lda, B, ldb)
    bound = np.repeat(bound.T.ravel(), 2) if np.iscomplexobj(ref) else bound.T.ravel()
    assert np.all(diff <= 1e-25 * (bound + 1e-300)), float(np.max(diff / (bound + 1e-300)))
    # the hi parts are the correctly rounded sums up to an ulp
    assert np.all(np.abs(gh - rh) <= 2.3e-16 * np.abs(rh) + 1e-25 * bound + 1e-300)


def test_dd_edge_sizes(spla_lib):
    """k = 0 gives zeros; m = 0 or n = 0 writes nothing; bad arguments are rejected."""
    import torch
    hi = torch.full((12,), 7.0, dtype=torch.float64, device="cuda")
    A = torch.ones(12, dtype=torch.float64, device="cuda")
    assert spla_lib.gemm_dd(1, 1, 0, 3, 4, 0, A, 1, A, 1, hi, 3) == 0
    torch.cuda.synchronize()
    assert torch.all(hi == 0)
    hi.fill_(7.0)
    assert spla_lib.gemm_dd(1, 1, 0, 0, 4, 5, A, 5, A, 5, hi, 1) == 0
    torch.cuda.synchronize()
    assert torch.all(hi == 7.0)
    assert spla_lib.gemm_dd(1, 1, 0, 3, 4, 5, A, 4, A, 5, hi, 3) != 0  # lda < k
    assert spla_lib.gemm_dd(7, 1, 0, 3, 4, 5, A, 5, A, 5, hi, 3) != 0  # dtype
