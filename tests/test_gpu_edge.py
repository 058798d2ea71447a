"""Edge shapes on every contraction path, against the double-double oracle:
single rows and columns, k = 1, very long k with a 1 x 1 result, k not a
multiple of any tile or block, m or n = 0 (no-op: C bit-unchanged), and
leading dimensions far above the sizes. Bars: 1e-14 relative Frobenius for
double dtypes, 1e-6 for float dtypes."""
import numpy as np
import pytest

import oracle
import spla_b200 as spla
from inputs import buffer

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (1, 1, 1_000_003), (1, 517, 3001), (333, 1, 20000), (7, 5, 1),
          (129, 65, 127), (64, 64, 100_001)]
PATHS = [(np.complex128, spla.PATH_DMMA, 1e-14), (np.complex128, spla.PATH_OZAKI, 1e-14),
         (np.float64, spla.PATH_OZAKI, 1e-14), (np.complex64, spla.PATH_TF32X3, 1e-6),
         (np.float32, spla.PATH_TF32X3, 1e-6), (np.complex64, spla.PATH_OZAKI, 1e-6)]


def _run(dt, path, m, n, k, pad=0, seed=3):
    import torch
    lda = k + pad
    A = buffer(dt, lda, m, seed, "gauss_k", k)
    B = buffer(dt, lda, n, seed + 1, "gauss_k", k)
    ldc = m + pad
    C = buffer(dt, ldc, n, seed + 2, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 64, 64)
    opA = 2 if np.dtype(dt).kind == "c" else 1
    dC = torch.from_numpy(C).cuda()
    spla.pgemm_ssb(m, n, k, opA, 1.0, torch.from_numpy(A).cuda(), lda,
                   torch.from_numpy(B).cuda(), lda, 0.5, dC, ldc, 0, 0, d, ctx)
    got = dC.cpu().numpy()
    ref = C.copy()
    assert oracle.pgemm_ssb(m, n, k, opA, 1.0, A, lda, B, lda, 0.5, ref, ldc, 0, 0) == 0
    return C, got, ref, ldc


@pytest.mark.parametrize("dt,path,tol", PATHS)
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_edge_shapes(dt, path, tol, m, n, k):
    C0, got, ref, ldc = _run(dt, path, m, n, k)
    err = oracle.rel_fro(got, ref)
    assert err <= tol, err


@pytest.mark.parametrize("dt,path,tol", PATHS)
def test_large_leading_dimensions(dt, path, tol):
    m, n, k, pad = 37, 29, 5000, 4099
    C0, got, ref, ldc = _run(dt, path, m, n, k, pad=pad)
    blk = lambda x: x.reshape(n, ldc)[:, :m]
    assert oracle.rel_fro(blk(got), blk(ref)) <= tol
    assert np.array_equal(got.reshape(n, ldc)[:, m:], C0.reshape(n, ldc)[:, m:])


@pytest.mark.parametrize("dt,path,tol", PATHS)
@pytest.mark.parametrize("m,n", [(0, 16), (16, 0)])
def test_empty_result_leaves_c(dt, path, tol, m, n):
    import torch
    C = buffer(dt, 16, 16, 9, "uniform11")
    dC = torch.from_numpy(C).cuda()
    A = torch.zeros(64 * 16, dtype=dC.dtype, device="cuda")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 64, 64)
    opA = 2 if np.dtype(dt).kind == "c" else 1
    spla.pgemm_ssb(m, n, 64, opA, 1.0, A, 64, A, 64, 0.0, dC, 16, 0, 0, d, ctx)
    assert np.array_equal(dC.cpu().numpy(), C)
