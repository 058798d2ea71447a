"""3xTF32 path (float / complex float on TF32 tcgen05) against the
double-double oracle, bar 1e-6 relative Frobenius error.

Covers: complex A^H B and A^T B, real A^T B, partial tiles in both
dimensions, several k super-chunks and FP32 drain chunks, alpha/beta with C
offsets and ldc padding (the rest of C bit-unchanged), k = 0, fill-mode tile
skipping, a double problem given the path (resolves to DMMA), and the failure
path of the bounded device waits (no GPU fault: the producer issues no
copies, every wait runs into a 50 ms bound)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
import spla_b200 as spla
from inputs import buffer

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(x).cuda()


def run_ssb(dt, m, n, k, opA, alpha=1.0, beta=0.0, ro=0, co=0, pad=0, fill=0, seed=11,
            dist="gauss_k", path=spla.PATH_TF32X3):
    A = buffer(dt, k + pad, m, seed, dist, k)
    B = buffer(dt, k + pad, n, seed + 1, dist, k)
    ldc = m + ro + pad
    C = buffer(dt, ldc, n + co, seed + 2, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    dC = _dev(C)
    spla.pgemm_ssbtr(m, n, k, opA, alpha, _dev(A), k + pad, _dev(B), k + pad, beta, dC, ldc, ro,
                     co, fill, d, ctx)
    got = dC.cpu().numpy()
    ref = C.copy()
    assert oracle.pgemm_ssb(m, n, k, opA, alpha, A, k + pad, B, k + pad, beta, ref, ldc, ro, co) == 0
    return C, got, ref, ldc


def block(x, ldc, m, n, ro, co):
    return x.reshape(-1, ldc)[co:co + n, ro:ro + m]


def test_path_resolution():
    assert spla.lib().splab_gemm_path(2, spla.PATH_TF32X3, 2, 0, 512, 512, 4096) == spla.PATH_TF32X3
    assert spla.lib().splab_gemm_path(0, spla.PATH_TF32X3, 1, 0, 512, 512, 4096) == spla.PATH_TF32X3
    # double dtypes are not handled by the path; op(A) = N is, through a k-major copy of A
    assert spla.lib().splab_gemm_path(3, spla.PATH_TF32X3, 2, 0, 512, 512, 4096) == spla.PATH_DMMA
    assert spla.lib().splab_gemm_path(2, spla.PATH_TF32X3, 0, 0, 512, 512, 4096) == spla.PATH_TF32X3


@pytest.mark.parametrize("dt,opA", [(np.complex64, 2), (np.complex64, 1), (np.float32, 1)])
def test_partial_tiles_many_chunks(dt, opA):
    # real-form k = 2k (complex) spans several 1024-real drain chunks and,
    # with 2 x 2 / 2 x 1 tiles, several super-chunks
    m, n, k = 300, 150, 70000
    alpha = 0.5 + 0.25j if np.dtype(dt).kind == "c" else 0.5
    C0, got, ref, ldc = run_ssb(dt, m, n, k, opA, alpha, -1.0)
    err = oracle.rel_fro(got, ref)
    assert err <= 1e-6, err


@pytest.mark.parametrize("dt", [np.complex64, np.float32])
def test_uniform_entries(dt):
    # non-centred entries: large sums, relative error set by the split
    m, n, k = 129, 257, 20000
    C0, got, ref, ldc = run_ssb(dt, m, n, k, 2 if np.dtype(dt).kind == "c" else 1,
                                dist="uniform100")
    err = oracle.rel_fro(got, ref)
    assert err <= 1e-6, err


@pytest.mark.parametrize("dt,opA", [(np.complex64, 2), (np.float32, 1)])
def test_overlap_matrix(dt, opA):
    """S = A^H A: the diagonal sums are sign-coherent (|a|^2), the case where a
    long FP32 accumulation chain on the tensor cores loses accuracy."""
    m, k = 260, 120000
    A = buffer(dt, k, m, 31, "gauss_k", k)
    C = np.zeros(m * m, dt)
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_TF32X3)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    dA, dC = _dev(A), _dev(C)
    spla.pgemm_ssb(m, m, k, opA, 1.0, dA, k, dA, k, 0.0, dC, m, 0, 0, d, ctx)
    ref = C.copy()
    assert oracle.pgemm_ssb(m, m, k, opA, 1.0, A, k, A, k, 0.0, ref, m, 0, 0) == 0
    err = oracle.rel_fro(dC.cpu().numpy(), ref)
    assert err <= 1e-6, err


def test_alpha_beta_offsets_padding():
    m, n, k, ro, co = 70, 90, 20000, 3, 2
    alpha, beta = 0.5 - 1.25j, 0.75 + 0.5j
    C0, got, ref, ldc = run_ssb(np.complex64, m, n, k, 2, alpha, beta, ro, co, pad=5)
    gb, rb = block(got, ldc, m, n, ro, co), block(ref, ldc, m, n, ro, co)
    assert oracle.rel_fro(gb, rb) <= 1e-6
    mask = np.ones((n + co, ldc), bool)
    mask[co:co + n, ro:ro + m] = False
    assert np.array_equal(got.reshape(-1, ldc)[mask], C0.reshape(-1, ldc)[mask])


def test_k_zero_scales_c():
    m, n = 40, 30
    C0, got, ref, ldc = run_ssb(np.complex64, m, n, 0, 2, 1.0, 0.5 - 0.5j)
    assert oracle.rel_fro(got, ref) <= 1e-6


def test_fill_lower_triangle():
    m = n = 300
    k = 6000
    C0, got, ref, ldc = run_ssb(np.complex64, m, n, k, 2, fill=spla.FILL_MODE_LOWER)
    g, r = got.reshape(n, ldc).T[:m], ref.reshape(n, ldc).T[:m]
    c0 = C0.reshape(n, ldc).T[:m]
    tri = np.tril(np.ones((m, n), bool))
    assert oracle.rel_fro(g[tri], r[tri]) <= 1e-6
    off = ~tri
    ok = np.isclose(g[off], r[off], rtol=1e-5, atol=1e-6) | (g[off] == c0[off])
    assert ok.all()


def test_double_falls_back_to_dmma():
    m, n, k = 64, 48, 5000
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, k, 2)
    assert oracle.rel_fro(got, ref) <= 1e-14


def test_bounded_wait_failure_path():
    """The TF32 GEMM's barrier waits are bounded: with the test hook the
    producer issues no copies, the waits give up after 50 ms, the kernel frees
    its tensor memory and returns, and the call reports SPLA_GPU_LAUNCH_ERROR
    (SPLAB_ERR_TIMEOUT) without faulting; the context stays usable."""
    code = r"""
import sys, numpy as np, torch
sys.path[:0] = [%r, %r]
import spla_b200 as spla
m, n, k = 64, 64, 4096
A = torch.randn(m * k, dtype=torch.complex64, device='cuda')
B = torch.randn(n * k, dtype=torch.complex64, device='cuda')
C = torch.zeros(m * n, dtype=torch.complex64, device='cuda')
ctx = spla.Context(spla.PU_GPU); ctx.set_fp64_path(spla.PATH_TF32X3)
d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, 'R', 1, 1, 64, 64)
try:
    spla.pgemm_ssb(m, n, k, 2, 1.0, A, k, B, k, 0.0, C, m, 0, 0, d, ctx)
    print('NO_ERROR')
except spla.GPULaunchError:
    print('TIMEOUT_REPORTED')
ctx.set_fp64_path(spla.PATH_DMMA)
spla.pgemm_ssb(m, n, k, 2, 1.0, A, k, B, k, 0.0, C, m, 0, 0, d, ctx)
torch.cuda.synchronize()
print('DEVICE_OK')
""" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
       os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, SPLAB_TF32X3_STALL_TEST="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=300)
    assert "TIMEOUT_REPORTED" in out.stdout, out.stdout + out.stderr
    assert "DEVICE_OK" in out.stdout, out.stdout + out.stderr
