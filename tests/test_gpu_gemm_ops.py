"""Local gemm() over the full operation matrix: op(A), op(B) in {N, T, C}
(all nine pairs) for the four dtypes, sizes that are not multiples of any
tile, alpha/beta complex, padded leading dimensions, on the default path, the
FP64 DMMA path, the Ozaki path and the 3xTF32 path (float dtypes), against the
double-double oracle (1e-14 double, 1e-6 float). The tensor-core paths take
every op pair (op(B) in {T, C}, and op(A) = N on 3xTF32, through a k-major
copy of the operand): each forced path is checked to be the one that ran."""
import numpy as np
import pytest

import oracle
import spla_b200 as spla
from inputs import buffer

pytestmark = pytest.mark.gpu

DT = [(np.float64, 1e-14), (np.complex128, 1e-14), (np.float32, 1e-6), (np.complex64, 1e-6)]
OPS = [(a, b) for a in (0, 1, 2) for b in (0, 1, 2)]


@pytest.mark.parametrize("dt,tol", DT)
@pytest.mark.parametrize("path", [spla.PATH_AUTO, spla.PATH_DMMA, spla.PATH_OZAKI,
                                  spla.PATH_TF32X3])
def test_gemm_all_ops(dt, tol, path):
    import torch
    code = {np.float32: 0, np.float64: 1, np.complex64: 2, np.complex128: 3}[dt]
    if path == spla.PATH_TF32X3 and code in (1, 3):
        pytest.skip("3xTF32 takes float dtypes only")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = ((0.75 - 0.5j), (0.25 + 1.0j)) if cplx else (0.75, -1.25)
    for i, (opA, opB) in enumerate(OPS):
        m, n, k = 67, 45, 301
        if path in (spla.PATH_OZAKI, spla.PATH_TF32X3):
            assert spla.lib().splab_gemm_path(code, path, opA, opB, m, n, k) == path
        lda = (m if opA == 0 else k) + 3
        ldb = (k if opB == 0 else n) + 5
        ldc = m + 2
        A = buffer(dt, lda, k if opA == 0 else m, 40 + i, "uniform11")
        B = buffer(dt, ldb, n if opB == 0 else k, 60 + i, "uniform11")
        C = buffer(dt, ldc, n, 80 + i, "uniform11")
        dC = torch.from_numpy(C).cuda()
        spla.gemm(opA, opB, m, n, k, alpha, torch.from_numpy(A).cuda(), lda,
                  torch.from_numpy(B).cuda(), ldb, beta, dC, ldc, ctx)
        ref = C.copy()
        assert oracle.gemm(opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, ref, ldc) == 0
        got = dC.cpu().numpy()
        blk = lambda x: x.reshape(n, ldc)[:, :m]
        err = oracle.rel_fro(blk(got), blk(ref))
        assert err <= tol, (opA, opB, err)
        assert np.array_equal(got.reshape(n, ldc)[:, m:], C.reshape(n, ldc)[:, m:])
