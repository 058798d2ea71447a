"""Ozaki scheme II path (INT8 tcgen05) against the double-double oracle.

Covers: complex A^H B and A^T B (three real products per modulus), real
A^T B, partial tiles in both dimensions, several k-chunks (k > 124928), the
workspace reused by a second call, alpha/beta with C offsets and
ldc padding, k = 0, the modulus-count knob, the fill-mode tile skipping,
op(A) = N (pgemm_sbs and gemm: A copied k-major first) with one k-chunk (byte
residues) and several (int32 sums), more row tiles than one band of the unit
raster, the reconstruction staged through shared memory, rows of extreme
magnitude, NaN/Inf propagation, and the failure
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


def run_ssb(dt, m, n, k, opA, alpha=1.0, beta=0.0, ro=0, co=0, pad=0, fill=0, moduli=0,
            seed=1, dist="gauss_k", path=spla.PATH_OZAKI, cols=None):
    A = buffer(dt, k + pad, m, seed, dist, k)
    B = buffer(dt, k + pad, n, seed + 1, dist, k)
    ldc = m + ro + pad
    C = buffer(dt, ldc, n + co, seed + 2, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path, moduli)
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


@pytest.mark.parametrize("opA", [2, 1])
def test_complex_multi_chunk_partial_tiles(opA):
    m, n, k = 300, 150, 150000  # rows of 150016 bytes -> 2 k-chunks; partial tiles
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, k, opA)
    err = oracle.rel_fro(got, ref)
    assert err <= 1e-14, err


@pytest.mark.parametrize("dt,opA", [(np.complex64, 2), (np.complex64, 1), (np.float32, 1)])
def test_float_dtypes(dt, opA):
    """Float inputs through the Ozaki path (9 moduli by default): the float
    result is within 1e-6 of the double-double oracle rounded to float."""
    m, n, k = 260, 140, 90000
    C0, got, ref, ldc = run_ssb(dt, m, n, k, opA, 0.5 + 0.25j if np.dtype(dt).kind == "c" else 0.5,
                                -1.0, dist="gauss_k")
    assert oracle.rel_fro(got, ref) <= 1e-6


@pytest.mark.parametrize("nt", ["1", "2"])
def test_pair_tile_widths(nt, monkeypatch):
    """Both INT8 GEMM tile widths (CTA pair 256 x 256 and 256 x 512) on a
    problem with partial tiles in both dimensions and two k-chunks."""
    monkeypatch.setenv("SPLAB_OZAKI_NT", nt)
    m, n, k = 333, 291, 130000  # residue rows of 130048 bytes -> 2 chunks
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, k, 2)
    assert oracle.rel_fro(got, ref) <= 1e-14


def test_real_double():
    m, n, k = 200, 330, 70000
    C0, got, ref, ldc = run_ssb(np.float64, m, n, k, 1, dist="uniform11")
    assert oracle.rel_fro(got, ref) <= 1e-14


def test_alpha_beta_offsets_padding():
    m, n, k, ro, co = 70, 90, 20000, 3, 2
    alpha, beta = 0.5 - 1.25j, 0.75 + 0.5j
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, k, 2, alpha, beta, ro, co, pad=5)
    gb, rb = block(got, ldc, m, n, ro, co), block(ref, ldc, m, n, ro, co)
    assert oracle.rel_fro(gb, rb) <= 1e-14
    # everything outside the block is bit-unchanged
    mask = np.ones((n + co, ldc), bool)
    mask[co:co + n, ro:ro + m] = False
    assert np.array_equal(got.reshape(-1, ldc)[mask], C0.reshape(-1, ldc)[mask])


def test_k_zero_scales_c():
    m, n = 40, 30
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, 0, 2, 1.0, 0.5 - 0.5j)
    assert oracle.rel_fro(got, ref) <= 1e-15


@pytest.mark.parametrize("moduli,bar", [(16, 1e-14), (14, 1e-13), (12, 1e-9)])
def test_modulus_count(moduli, bar):
    m, n, k = 130, 70, 30000
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, k, 2, moduli=moduli)
    assert oracle.rel_fro(got, ref) <= bar


def test_modulus_count_out_of_range_rejected():
    ctx = spla.Context(spla.PU_GPU)
    with pytest.raises(spla.InvalidParameterError):
        ctx.set_fp64_path(spla.PATH_OZAKI, 17)
    with pytest.raises(spla.InvalidParameterError):
        ctx.set_fp64_path(spla.PATH_OZAKI, 5)


@pytest.mark.parametrize("m", [300, 512])
def test_fill_lower_triangle(m):
    n = m
    k = 6000
    C0, got, ref, ldc = run_ssb(np.complex128, m, n, k, 2, fill=spla.FILL_MODE_LOWER)
    g, r = got.reshape(n, ldc).T[:m], ref.reshape(n, ldc).T[:m]
    c0 = C0.reshape(n, ldc).T[:m]
    tri = np.tril(np.ones((m, n), bool))
    assert oracle.rel_fro(g[tri], r[tri]) <= 1e-14
    off = ~tri
    ok = np.isclose(g[off], r[off], rtol=1e-12, atol=1e-14) | (g[off] == c0[off])
    assert ok.all()


@pytest.mark.parametrize("dt,tol", [(np.complex128, 1e-14), (np.float64, 1e-14),
                                    (np.complex64, 1e-6), (np.float32, 1e-6)])
def test_sbs_op_n(dt, tol):
    """pgemm_sbs (C = alpha A B + beta C, A an m-major stripe) on the Ozaki
    path: ragged sizes, padded leading dimensions, one k-chunk."""
    cplx = np.dtype(dt).kind == "c"
    mloc, n, k, pad = 701, 130, 900, 3
    alpha, beta = ((0.5 - 0.25j), (1.0 + 0.5j)) if cplx else (0.5, 1.0)
    A = buffer(dt, mloc + pad, k, 31, "gauss_k", k)
    B = buffer(dt, k + pad, n, 32, "uniform11")
    C = buffer(dt, mloc + pad, n, 33, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_OZAKI)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    dC = _dev(C)
    spla.pgemm_sbs(mloc, n, k, alpha, _dev(A), mloc + pad, _dev(B), k + pad, 0, 0, d, beta, dC,
                   mloc + pad, ctx)
    got = dC.cpu().numpy()
    ref = C.copy()
    assert oracle.pgemm_sbs(mloc, n, k, alpha, A, mloc + pad, B, k + pad, 0, 0, beta, ref,
                            mloc + pad) == 0
    blk = lambda x: x.reshape(n, mloc + pad)[:, :mloc]  # noqa: E731
    assert oracle.rel_fro(blk(got), blk(ref)) <= tol
    assert np.array_equal(got.reshape(n, mloc + pad)[:, mloc:], C.reshape(n, mloc + pad)[:, mloc:])


def test_gemm_op_n_multi_chunk():
    """gemm(N, N) on the Ozaki path with k > 124928 (two k-chunks: the
    residues are int32 sums) and a padded A."""
    m, n, k, lda = 90, 40, 130000, 97
    alpha, beta = 1.0 - 0.5j, -0.5 + 0.25j
    A = buffer(np.complex128, lda, k, 41, "gauss_k", k)
    B = buffer(np.complex128, k, n, 42, "gauss_k", k)
    C = buffer(np.complex128, m, n, 43, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_OZAKI)
    dC = _dev(C)
    spla.gemm(0, 0, m, n, k, alpha, _dev(A), lda, _dev(B), k, beta, dC, m, ctx)
    ref = C.copy()
    assert oracle.gemm(0, 0, m, n, k, alpha, A, lda, B, k, beta, ref, m) == 0
    assert oracle.rel_fro(dC.cpu().numpy(), ref) <= 1e-14


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_tall_banded_raster(dt):
    """More row tiles than one band (8 x 256 rows) with a partial last band,
    on the ssb (op(A) = T/C) and gemm op(A) = N forms: every tile of the
    banded unit order is computed once."""
    import torch
    cplx = np.dtype(dt).kind == "c"
    m, n, k = 2600, 300, 400
    C0, got, ref, ldc = run_ssb(dt, m, n, k, 2 if cplx else 1, dist="uniform11")
    assert oracle.rel_fro(got, ref) <= 1e-14
    A = buffer(dt, m, k, 51, "uniform11")
    B = buffer(dt, k, n, 52, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_OZAKI)
    dC = torch.zeros(m * n, dtype=torch.complex128 if cplx else torch.float64, device="cuda")
    spla.gemm(0, 0, m, n, k, 1.0, _dev(A), m, _dev(B), k, 0.0, dC, m, ctx)
    ref = np.zeros(m * n, dtype=dt)
    assert oracle.gemm(0, 0, m, n, k, 1.0, A, m, B, k, 0.0, ref, m) == 0
    assert oracle.rel_fro(dC.cpu().numpy(), ref) <= 1e-14


@pytest.mark.parametrize("dt,tol", [(np.complex128, 1e-14), (np.float32, 1e-6)])
def test_fill_lower_wide_tile(dt, tol, monkeypatch):
    """Lower fill mode on the 256 x 512 pair tile (the default for long units,
    forced here): every element of the triangle is computed, the rest is
    either computed or unchanged."""
    monkeypatch.setenv("SPLAB_OZAKI_NT", "2")
    m = n = 520
    k = 16500  # residue rows of 16512 bytes: 129 k-blocks
    C0, got, ref, ldc = run_ssb(dt, m, n, k, 2 if np.dtype(dt).kind == "c" else 1,
                                fill=spla.FILL_MODE_LOWER)
    g, r = got.reshape(n, ldc).T[:m], ref.reshape(n, ldc).T[:m]
    c0 = C0.reshape(n, ldc).T[:m]
    tri = np.tril(np.ones((m, n), bool))
    assert oracle.rel_fro(g[tri], r[tri]) <= tol
    off = ~tri
    ok = np.isclose(g[off], r[off], rtol=1e-5, atol=1e-7) | (g[off] == c0[off])
    assert ok.all()


@pytest.mark.parametrize("dt,tol,m,moduli", [
    (np.complex128, 1e-14, 3088, 0), (np.float64, 1e-14, 1040, 0),
    (np.complex64, 1e-6, 2064, 0), (np.float32, 1e-6, 1056, 0), (np.complex128, 1e-9, 2064, 12)])
def test_staged_reconstruction(dt, tol, m, moduli):
    """Byte residues with m % 16 == 0 take the reconstruction staged through
    shared memory: several blocks of 1024 rows with a partial last one, alpha
    and beta both active, the default and a non-default modulus count."""
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = ((0.5 + 0.25j), (-1.0 + 0.5j)) if cplx else (0.5, -1.0)
    C0, got, ref, ldc = run_ssb(dt, m, 70, 500, 2 if cplx else 1, alpha, beta, moduli=moduli)
    assert oracle.rel_fro(got, ref) <= tol


@pytest.mark.parametrize("dt", [np.complex128, np.float64])
def test_workspace_reused_across_calls(dt):
    """Two multi-chunk calls (int32 residue sums) through one context reuse its
    workspace: the sums of the second call must start from zero in every
    product plane, so both results match the oracle."""
    import torch
    cplx = np.dtype(dt).kind == "c"
    m, n, k = 130, 70, 140000  # residue rows of 140032 bytes: 2 k-chunks
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_OZAKI)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    for seed in (71, 72):
        A = buffer(dt, k, m, seed, "gauss_k", k)
        B = buffer(dt, k, n, seed + 10, "gauss_k", k)
        dC = torch.zeros(m * n, dtype=torch.complex128 if cplx else torch.float64, device="cuda")
        spla.pgemm_ssb(m, n, k, 2 if cplx else 1, 1.0, _dev(A), k, _dev(B), k, 0.0, dC, m, 0, 0,
                       d, ctx)
        ref = np.zeros(m * n, dtype=dt)
        assert oracle.pgemm_ssb(m, n, k, 2 if cplx else 1, 1.0, A, k, B, k, 0.0, ref, m, 0, 0) == 0
        assert oracle.rel_fro(dC.cpu().numpy(), ref) <= 1e-14, seed


@pytest.mark.parametrize("dt", [np.complex128, np.float64])
def test_extreme_row_magnitudes(dt):
    """Rows of A scaled to 1e-170 and 1e150 (their squared norms would
    underflow or overflow in plain double): each row of C matches the oracle
    to 1e-14 of its own norm."""
    import torch
    cplx = np.dtype(dt).kind == "c"
    m, n, k = 64, 40, 3000
    A = buffer(dt, k, m, 81, "gauss_k", k)
    B = buffer(dt, k, n, 82, "gauss_k", k)
    scale = np.ones(m)
    scale[:16] = 1e-170
    scale[16:32] = 1e150
    A = np.ascontiguousarray((A.reshape(m, k) * scale[:, None]).ravel())
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_OZAKI)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    dC = torch.zeros(m * n, dtype=torch.complex128 if cplx else torch.float64, device="cuda")
    op = 2 if cplx else 1
    spla.pgemm_ssb(m, n, k, op, 1.0, _dev(A), k, _dev(B), k, 0.0, dC, m, 0, 0, d, ctx)
    ref = np.zeros(m * n, dtype=dt)
    assert oracle.pgemm_ssb(m, n, k, op, 1.0, A, k, B, k, 0.0, ref, m, 0, 0) == 0
    g, r = dC.cpu().numpy().reshape(n, m).T, ref.reshape(n, m).T
    for i in range(m):
        mx = np.abs(r[i]).max()  # norm without underflow or overflow of the squares
        assert np.abs(g[i] - r[i]).max() <= 1e-14 * mx * np.linalg.norm(r[i] / mx), i


def test_nan_and_inf_propagate():
    """A NaN in row 3 of A and an infinity in column 5 of B: that row and
    column of C come out NaN, every other element matches the oracle."""
    import torch
    dt = np.complex128
    m, n, k = 40, 24, 2000
    A = buffer(dt, k, m, 91, "gauss_k", k)
    B = buffer(dt, k, n, 92, "gauss_k", k)
    A[3 * k + 17] = complex(np.nan, 0.0)
    B[5 * k + 100] = complex(np.inf, 1.0)
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_OZAKI)
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    dC = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    spla.pgemm_ssb(m, n, k, 2, 1.0, _dev(A), k, _dev(B), k, 0.0, dC, m, 0, 0, d, ctx)
    g = dC.cpu().numpy().reshape(n, m).T
    assert np.isnan(g[3, :]).all() and np.isnan(g[:, 5]).all()
    A2, B2 = A.copy(), B.copy()
    A2[3 * k + 17] = 0.0
    B2[5 * k + 100] = 0.0
    ref = np.zeros(m * n, dtype=dt)
    assert oracle.pgemm_ssb(m, n, k, 2, 1.0, A2, k, B2, k, 0.0, ref, m, 0, 0) == 0
    r = ref.reshape(n, m).T
    mask = np.ones((m, n), bool)
    mask[3, :] = False
    mask[:, 5] = False
    assert oracle.rel_fro(g[mask], r[mask]) <= 1e-14


@pytest.mark.parametrize("dt,m,n,k,opA", [(np.complex128, 130, 70, 140000, 2),
                                          (np.float64, 200, 120, 3000, 1)])
def test_single_cta_gemm(dt, m, n, k, opA, monkeypatch):
    """The single-CTA INT8 GEMM kept beside the CTA-pair one
    (SPLAB_OZAKI_GEMM=1sm): two k-chunks (int32 sums) and one (byte
    residues)."""
    monkeypatch.setenv("SPLAB_OZAKI_GEMM", "1sm")
    C0, got, ref, ldc = run_ssb(dt, m, n, k, opA)
    assert oracle.rel_fro(got, ref) <= 1e-14


def test_bounded_wait_failure_path():
    """The INT8 GEMM's barrier waits are bounded: with the test hook the
    producer issues no copies, the waits give up after 50 ms, the kernel frees
    its tensor memory and returns, and the call reports SPLA_GPU_LAUNCH_ERROR
    (SPLAB_ERR_TIMEOUT) without faulting; the context stays usable."""
    code = r"""
import sys, numpy as np, torch
sys.path[:0] = [%r, %r]
import spla_b200 as spla
m, n, k = 64, 64, 4096
A = torch.randn(m * k, dtype=torch.complex128, device='cuda')
B = torch.randn(n * k, dtype=torch.complex128, device='cuda')
C = torch.zeros(m * n, dtype=torch.complex128, device='cuda')
ctx = spla.Context(spla.PU_GPU); ctx.set_fp64_path(spla.PATH_OZAKI)
d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, 'R', 1, 1, 64, 64)
try:
    spla.pgemm_ssb(m, n, k, 2, 1.0, A, k, B, k, 0.0, C, m, 0, 0, d, ctx)
    print('NO_ERROR')
except spla.GPULaunchError:
    print('TIMEOUT_REPORTED')
# the device is still usable afterwards
ctx.set_fp64_path(spla.PATH_DMMA)
spla.pgemm_ssb(m, n, k, 2, 1.0, A, k, B, k, 0.0, C, m, 0, 0, d, ctx)
torch.cuda.synchronize()
print('DEVICE_OK')
""" % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
       os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, SPLAB_OZAKI_STALL_TEST="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=300)
    assert "TIMEOUT_REPORTED" in out.stdout, out.stdout + out.stderr
    assert "DEVICE_OK" in out.stdout, out.stdout + out.stderr


@pytest.mark.parametrize("m,n,k,opA,pad", [(300, 150, 150000, 2, 0), (257, 129, 1000, 1, 3),
                                           (40, 24, 3000, 2, 1), (513, 70, 769, 0, 0),
                                           (128, 1024, 250000, 2, 0)])
def test_tensor_core_slicer_matches_fp32_slicer(m, n, k, opA, pad):
    """Complex double rows are sliced with the digit sums on the INT8 tensor
    cores (oz_slice_tc); SPLAB_OZAKI_SLICE_TC=0 selects the FP32 digit-sum
    slicer. Both produce the same symmetric residues, so C is bit-identical:
    unit tails (k not a multiple of 768), residue rows padded to 128, partial
    groups, op(A) = N (the k-major copy), both signs of the sum plane, and
    several k-chunks."""
    import torch
    dt = np.complex128
    lda = (m if opA == 0 else k) + pad
    A = buffer(dt, lda, k if opA == 0 else m, 31, "gauss_k", k)
    B = buffer(dt, k + pad, n, 32, "gauss_k", k)
    C = buffer(dt, m + pad, n, 33, "uniform11")
    out = []
    for tc in ("1", "0"):
        os.environ["SPLAB_OZAKI_SLICE_TC"] = tc
        try:
            ctx = spla.Context(spla.PU_GPU)
            ctx.set_fp64_path(spla.PATH_OZAKI)
            dC = _dev(C)
            spla.gemm(opA, 0, m, n, k, 0.5 - 0.25j, _dev(A), lda, _dev(B), k + pad, 1.5, dC,
                      m + pad, ctx)
            torch.cuda.synchronize()
            out.append(dC.cpu().numpy())
        finally:
            os.environ.pop("SPLAB_OZAKI_SLICE_TC", None)
    assert np.array_equal(out[0], out[1])
    # accuracy against the device double-double product (k up to 250000)
    R = torch.zeros(n * (m + pad), dtype=torch.complex128, device="cuda")
    assert spla.gemm_dd(3, opA, 0, m, n, k, _dev(A), lda, _dev(B), k + pad, R, m + pad) == 0
    torch.cuda.synchronize()
    ref = ((0.5 - 0.25j) * R.cpu().numpy() + 1.5 * C).reshape(n, m + pad)[:, :m]
    assert oracle.rel_fro(out[0].reshape(n, m + pad)[:, :m], ref) <= 1e-14


@pytest.mark.parametrize("dt,m,n,k,opA,fill,moduli,nan", [
    (np.complex128, 3088, 70, 500, 2, 0, 0, False),     # partial last block of 128 rows
    (np.complex128, 400, 130, 3000, 1, 0, 0, False),    # A^T B: the other signs of Im
    (np.complex128, 520, 520, 16500, 2, spla.FILL_MODE_LOWER, 0, False),
    (np.complex128, 2064, 70, 500, 2, 0, 12, False),    # non-default modulus count
    (np.complex128, 256, 200, 1000, 2, 0, 0, True),     # a NaN row of A and of B
    (np.float64, 1040, 70, 500, 1, 0, 0, False),
    (np.complex64, 2064, 70, 500, 2, 0, 0, False),
    (np.float32, 1056, 70, 500, 1, 0, 0, False),
    (np.complex128, 300, 150, 1000, 2, 0, 0, False),    # m % 16 != 0: plain kernel
    (np.float32, 77, 50, 500, 1, 0, 0, False),          # m below one block of 128 rows
])
def test_tensor_core_reconstruction_matches_staged(dt, m, n, k, opA, fill, moduli, nan):
    """Byte residues (one k-chunk) with m % 16 == 0 and m >= 128 are
    reconstructed with the CRT sums on the INT8 tensor cores
    (oz_reconstruct_tc); SPLAB_OZAKI_RECON_TC=0 selects the staged CUDA-core
    kernel (the last two cases take the plain kernel either way). Both reduce
    the same congruence class to the same limbs, so C is bit-identical (bytes
    compared, NaN included); both are also checked against the oracle."""
    import torch
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = ((0.5 + 0.25j), (-1.0 + 0.5j)) if cplx else (0.5, -1.0)
    A = buffer(dt, k, m, 41, "gauss_k", k)
    B = buffer(dt, k, n, 42, "gauss_k", k)
    if nan:
        A[k * 7 + 3] = np.nan
        B[k * 5 + 1] = np.nan
    C = buffer(dt, m, n, 43, "uniform11")
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 128, 128)
    out = []
    for tc in ("1", "0"):
        os.environ["SPLAB_OZAKI_RECON_TC"] = tc
        try:
            ctx = spla.Context(spla.PU_GPU)
            ctx.set_fp64_path(spla.PATH_OZAKI, moduli)
            dC = _dev(C)
            spla.pgemm_ssbtr(m, n, k, opA, alpha, _dev(A), k, _dev(B), k, beta, dC, m, 0, 0,
                             fill, d, ctx)
            torch.cuda.synchronize()
            out.append(dC.cpu().numpy())
        finally:
            os.environ.pop("SPLAB_OZAKI_RECON_TC", None)
    assert np.array_equal(out[0].view(np.uint8), out[1].view(np.uint8))
    ref = C.copy()
    assert oracle.pgemm_ssb(m, n, k, opA, alpha, A, k, B, k, beta, ref, m, 0, 0) == 0
    g, r = out[0].reshape(n, m).T, ref.reshape(n, m).T
    sel = np.tril(np.ones((m, n), bool)) if fill else np.ones((m, n), bool)
    if nan:
        bad = np.zeros((m, n), bool)
        bad[7, :] = True
        bad[:, 5] = True
        assert np.isnan(g[bad]).all()
        sel &= ~bad
    tol = 1e-9 if moduli else (1e-14 if np.dtype(dt).itemsize >= 16 or dt == np.float64 else 1e-6)
    assert oracle.rel_fro(g[sel], r[sel]) <= tol


@pytest.mark.parametrize("dt,opA,opB,m,n,k,pad,offset", [
    ("complex128", 0, 0, 65536 + 37, 48, 999, 0, False),  # many rows, ragged m and k
    ("complex128", 0, 0, 70000, 40, 1000, 5, True),       # padded lda, base 8 bytes off 16
    ("float64", 0, 0, 65536 + 9, 40, 1500, 3, False),
    ("complex64", 0, 0, 66000, 40, 700, 0, False),
    ("float32", 0, 0, 65600, 36, 900, 1, False),
    ("complex128", 0, 0, 300, 200, 40000, 2, False),      # few rows: k-sliced norms
    ("complex128", 2, 1, 257, 300, 20000, 1, False),      # op(B) = T in place
    ("complex128", 1, 2, 128, 260, 3000, 0, True),        # op(B) = C: conjugated on load
    ("complex128", 0, 2, 200, 70001, 600, 0, False),      # both in place, many B rows
    ("float64", 1, 1, 190, 210, 30000, 2, False),
    ("complex64", 0, 2, 150, 170, 20000, 0, False),
    ("float32", 0, 1, 100, 90, 50000, 0, False),
    ("float64", 0, 0, 4, 8, 4_000_000, 0, False),         # 4096 k-slices (the grid's limit)
])
def test_in_place_operands(dt, opA, opB, m, n, k, pad, offset):
    """op(A) = N and op(B) = T or C are read in place (m- and n-major rows):
    row norms along the rows (k-sliced and combined when the rows are few)
    and residues through a transposing shared-memory tile, conjugated on load
    for op(B) = C; no k-major copy of either operand. Checked against the
    device double-double product, with alpha and beta, ragged sizes, padded
    leading dimensions and (complex double) a base address only 8-byte
    aligned (the scalar-load variant)."""
    import torch
    cplx = dt.startswith("complex")
    rt = torch.float64 if dt in ("complex128", "float64") else torch.float32
    r = 2 if cplx else 1
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    s = (1.0 / (r * k)) ** 0.5
    lda = (m if opA == 0 else k) + pad
    ldb = (k if opB == 0 else n) + pad
    acols = k if opA == 0 else m
    bcols = n if opB == 0 else k
    Abuf = torch.randn(r * lda * acols + 2, dtype=rt, device="cuda", generator=g) * s
    A = Abuf[1:] if offset else Abuf  # complex double at one real off: 8 bytes off 16
    B = torch.randn(r * ldb * bcols, dtype=rt, device="cuda", generator=g) * s
    C0 = torch.rand(r * m * n, dtype=rt, device="cuda", generator=g) * 2 - 1
    alpha, beta = ((0.5 - 0.25j), (1.0 + 0.5j)) if cplx else (0.5, -1.0)
    C = C0.clone()
    ws_bytes = spla.splab_gemm_workspace_size(dt, spla.PATH_OZAKI, opA, opB, m, n, k)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    assert spla.lib().splab_gemm_path(spla._dtype_of(dtype=dt), spla.PATH_OZAKI, opA, opB, m, n,
                                      k) == spla.PATH_OZAKI
    rc = spla.splab_gemm(dt, spla.PATH_OZAKI, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C,
                         m, workspace=ws, workspace_bytes=ws_bytes)
    assert rc == 0
    Rdt = torch.complex128 if cplx else torch.float64
    R = torch.zeros(m * n, dtype=Rdt, device="cuda")
    Ad = A.double() if rt == torch.float32 else A
    Bd = B.double() if rt == torch.float32 else B
    assert spla.gemm_dd("complex128" if cplx else "float64", opA, opB, m, n, k, Ad, lda, Bd, ldb,
                        R, m) == 0
    torch.cuda.synchronize()
    if cplx:
        got = torch.view_as_complex(C.double().reshape(-1, 2))
        c0 = torch.view_as_complex(C0.double().reshape(-1, 2))
    else:
        got, c0 = C.double(), C0.double()
    ref = alpha * R + beta * c0
    err = float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref))
    tol = 1e-14 if rt == torch.float64 else 1e-6
    assert err <= tol, err


def test_in_place_non_finite_and_extreme_rows():
    """The k-sliced in-place row norms (op(A) = N, op(B) = T; few rows, so the
    k range is sliced and the partial sums combined) keep the k-major path's
    semantics: a NaN or an infinity anywhere in a row makes that row's results
    NaN, and rows of magnitude 1e300 or 1e-300 scale without overflow or
    underflow (checked against the device double-double product)."""
    import torch
    m, n, k = 96, 80, 30000
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    s = (1.0 / (2 * k)) ** 0.5
    A = torch.randn(m * k, dtype=torch.complex128, device="cuda", generator=g) * s  # m x k
    B = torch.randn(n * k, dtype=torch.complex128, device="cuda", generator=g) * s  # n x k
    Av = A.view(k, m)  # element (i, kk) at kk * m + i
    Bv = B.view(k, n)
    Av[:, 3] *= 1e300
    Av[:, 4] *= 1e-300
    Bv[:, 6] *= 1e-300  # (3, 6) meets a 1e300 row: about 1
    Av[20000, 9] = complex(float("nan"), 0.0)   # late in the row: another k-slice
    Bv[25000, 11] = complex(0.0, float("inf"))
    C = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    ws_bytes = spla.splab_gemm_workspace_size("complex128", spla.PATH_OZAKI, 0, 1, m, n, k)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    assert spla.splab_gemm("complex128", spla.PATH_OZAKI, 0, 1, m, n, k, 1.0, A, m, B, n, 0.0,
                           C, m, workspace=ws, workspace_bytes=ws_bytes) == 0
    R = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    assert spla.gemm_dd("complex128", 0, 1, m, n, k, A, m, B, n, R, m) == 0
    torch.cuda.synchronize()
    got = C.view(n, m).T.cpu().numpy()
    ref = R.view(n, m).T.cpu().numpy()
    bad = np.zeros((m, n), bool)
    bad[9, :] = True
    bad[:, 11] = True
    assert np.isnan(got[bad]).all()
    ok = ~bad

    def rel(x, r):  # relative Frobenius error, scaled first (rows near 1e300)
        sc = np.abs(r).max()
        return oracle.rel_fro(x / sc, r / sc)

    # the extreme rows and column on their own scale, then the ordinary block
    for sel in (np.s_[3, :], np.s_[4, :], np.s_[:, 6]):
        keep = ok[sel]
        assert rel(got[sel][keep], ref[sel][keep]) <= 1e-14
    rows = np.r_[0:3, 5:m]
    block_ok = ok[rows][:, [c for c in range(n) if c != 6]]
    gb = got[rows][:, [c for c in range(n) if c != 6]]
    rb = ref[rows][:, [c for c in range(n) if c != 6]]
    assert rel(gb[block_ok], rb[block_ok]) <= 1e-14


@pytest.mark.parametrize("dt,opA,m,n,k,pad,offset", [
    ("complex128", 2, 136, 72, 70000, 0, False),   # 2k = 140000 reals per row
    ("complex128", 1, 130, 66, 66000, 3, True),    # A^T B; padded, 8 bytes off 16
    ("float64", 1, 120, 70, 140000, 0, False),
    ("float64", 1, 97, 33, 131072, 5, True),       # the shortest rows that take it
    ("complex64", 2, 140, 64, 70000, 0, False),
    ("float32", 1, 100, 60, 150000, 2, False),
])
def test_one_pass_row_scaling_matches_two_pass(dt, opA, m, n, k, pad, offset):
    """Long k-major rows take their scale exponents from a sample of each row
    (16 evenly spread runs), checked after slicing by the sum of squares of
    the scaled values; rows the sample misjudges get the exact norm and are
    sliced again; rows whose estimate lies next to a power of two take the
    exact norm at once. Rows built to defeat the sample (all their weight
    outside it, a NaN or an infinity outside it, zero rows, norms exactly a
    power of two, rows normalised to 1, 1e300 and 1e-300, a steep profile
    along k) end with the two-pass
    exponents and residues: C is bit-identical to SPLAB_OZAKI_ONEPASS=0 (bytes
    compared, NaN included), the one-pass sequence is seen to run (its
    fix-up phase event is recorded), and the finite part of C matches the
    device double-double product; with padded leading dimensions and base
    addresses only 8 bytes aligned (scalar loads) as well."""
    import ctypes as ct
    import torch
    cplx = dt.startswith("complex")
    rt = torch.float64 if dt in ("complex128", "float64") else torch.float32
    r = 2 if cplx else 1
    K2 = r * k
    g = torch.Generator(device="cuda")
    g.manual_seed(13)
    s = (1.0 / K2) ** 0.5
    ld = k + pad
    Abuf = torch.randn(r * ld * m + 1, dtype=rt, device="cuda", generator=g) * s
    Bbuf = torch.randn(r * ld * n + 1, dtype=rt, device="cuda", generator=g) * s
    A = Abuf[1:] if offset else Abuf[:-1]  # one real off: 8 (4) bytes off 16
    B = Bbuf[1:] if offset else Bbuf[:-1]
    # row i of op(A) / column j of op(B): K2 reals of a row of r * ld
    Ar, Br = A.view(m, r * ld)[:, :K2], B.view(n, r * ld)[:, :K2]
    # the sample: 16 runs of about K2 / 256 reals starting K2 // 16 apart, so
    # real K2 // 32 lies outside every run
    out = K2 // 16 // 2
    big = 1e30 if rt == torch.float64 else 1e15
    Ar[0].zero_(); Ar[0, out] = 3.0                      # all weight outside the sample
    Ar[1, out + 1] = 1e6                                 # one large element outside it
    Ar[2, out] = float("nan")
    Ar[3, out + 2] = float("inf")
    Ar[4].zero_()                                         # zero row
    Ar[5].zero_(); Ar[5, 0] = 2.0 ** 40                  # norm exactly a power of two
    Ar[6].zero_(); Ar[6, 0] = 0.6; Ar[6, 1] = 0.8         # norm 1 up to rounding
    Ar[7] *= 1e300 if rt == torch.float64 else 1e30
    Ar[8] *= 1e-300 if rt == torch.float64 else 1e-30
    Ar[9] *= torch.exp(-20.0 * torch.arange(K2, device="cuda", dtype=rt) / K2)  # steep decay
    Ar[10, : K2 // 2] *= 1e-8                            # small prefix, large rest
    Ar[11, K2 // 2:] *= big                              # large end
    # rows normalised to 1 and to 2^-3: estimates next to a power of two
    # take the exact norm at once
    Ar[12:40] /= torch.linalg.vector_norm(Ar[12:40], dim=1, keepdim=True)
    Ar[30:40] *= 0.125
    Br[0].zero_(); Br[0, out] = -1.0
    Br[1, out + 3] = float("nan")
    Br[2].zero_()
    Br[3] *= 1e-300 if rt == torch.float64 else 1e-30
    Br[4, K2 - 1] = 1e8
    C0 = torch.rand(r * m * n, dtype=rt, device="cuda", generator=g) * 2 - 1
    alpha, beta = ((0.5 - 0.25j), (1.0 + 0.5j)) if cplx else (0.5, -1.0)
    ws_bytes = spla.splab_gemm_workspace_size(dt, spla.PATH_OZAKI, opA, 0, m, n, k)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    L = spla.lib()
    nphase = 20
    st = torch.cuda.Stream()
    outs, redo = [], []
    for onepass in ("1", "0"):
        os.environ["SPLAB_OZAKI_ONEPASS"] = onepass
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * nphase)]
        for e in ev:
            e.record(st)
        st.synchronize()
        handles = (ct.c_void_p * (2 * nphase))(*[e.cuda_event for e in ev])
        C = C0.clone()
        torch.cuda.synchronize()
        L.splab_set_phase_events(handles, nphase)
        try:
            rc = spla.splab_gemm(dt, spla.PATH_OZAKI, opA, 0, m, n, k, alpha, A, ld, B, ld, beta, C,
                                 m, workspace=ws, workspace_bytes=ws_bytes, stream=st.cuda_stream)
        finally:
            L.splab_set_phase_events(None, 0)
            os.environ.pop("SPLAB_OZAKI_ONEPASS", None)
        assert rc == 0
        st.synchronize()
        outs.append(C.cpu().numpy())
        # phase 19 (the one-pass fix-up) ends after phase 18 (B's residues)
        # only when it ran; else its end event keeps the earlier record
        redo.append(ev[37].elapsed_time(ev[39]) if onepass == "1"
                    else ev[39].elapsed_time(ev[37]))
    assert redo[0] > 0.0 and redo[1] > 0.0, redo
    assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))
    # the finite part against the device double-double product
    Rdt = torch.complex128 if cplx else torch.float64
    R = torch.zeros(m * n, dtype=Rdt, device="cuda")
    Ad, Bd = A.double().clone(), B.double().clone()  # storage offset 0
    if cplx:
        Ad, Bd = torch.view_as_complex(Ad.view(-1, 2)), torch.view_as_complex(Bd.view(-1, 2))
    assert spla.gemm_dd("complex128" if cplx else "float64", opA, 0, m, n, k, Ad, ld, Bd, ld, R,
                        m) == 0
    torch.cuda.synchronize()
    c0 = C0.double().cpu().numpy()
    got = outs[0].astype(np.float64)
    if cplx:
        got = got.view(np.complex128)
        c0 = c0.view(np.complex128)
    ref = (alpha * R.cpu().numpy() + beta * c0).reshape(n, m).T
    got = got.reshape(n, m).T
    bad = np.zeros((m, n), bool)
    bad[[2, 3], :] = True
    bad[:, 1] = True
    assert np.isnan(got[bad]).all()
    # normwise: |C - ref| <= tol (|alpha| |a_i| |b_j| + |beta c0|), with the
    # norms taken without overflow (rows near 1e300)
    def norms(X, rows):  # NaN for the rows holding a NaN or an infinity
        x = X.double().view(rows, r * ld)[:, :K2].cpu().numpy()
        mx = np.abs(x).max(axis=1)
        mx[~((mx > 0) & np.isfinite(mx))] = 1.0
        with np.errstate(invalid="ignore"):
            return mx * np.linalg.norm(x / mx[:, None], axis=1)
    na, nb = norms(A, m), norms(B, n)
    tol = 1e-14 if rt == torch.float64 else 1e-6
    with np.errstate(invalid="ignore"):  # NaN bounds for the NaN rows
        bound = tol * (abs(alpha) * na[:, None] * nb[None, :] +
                       abs(beta) * np.abs(c0.reshape(n, m).T))
    ok = ~bad
    assert (np.abs(got - ref)[ok] <= bound[ok]).all()


@pytest.mark.parametrize("dt,opA,opB,m,n,k", [
    ("complex128", 0, 0, 150, 90, 70000),   # A read in place, B in one pass
    ("complex128", 2, 2, 120, 100, 66000),  # A in one pass, B read in place (conjugated)
    ("float64", 1, 1, 110, 96, 140000),
    ("complex64", 0, 0, 96, 130, 70000),
])
def test_one_pass_beside_an_operand_read_in_place(dt, opA, opB, m, n, k):
    """With one operand read in place (its norms k-sliced along m- or n-major
    rows) the other, k-major, is still scaled in one pass: C is bit-identical
    to SPLAB_OZAKI_ONEPASS=0, the fix-up phase runs, and C matches the device
    double-double product."""
    import ctypes as ct
    import torch
    cplx = dt.startswith("complex")
    rt = torch.float64 if dt in ("complex128", "float64") else torch.float32
    r = 2 if cplx else 1
    K2 = r * k
    g = torch.Generator(device="cuda")
    g.manual_seed(17)
    s = (1.0 / K2) ** 0.5
    A = torch.randn(r * k * m, dtype=rt, device="cuda", generator=g) * s
    B = torch.randn(r * k * n, dtype=rt, device="cuda", generator=g) * s
    lda, ldb = (m if opA == 0 else k), (k if opB == 0 else n)
    out = K2 // 32  # outside every sampled run
    if opA != 0:  # A k-major: rows of op(A) contiguous
        Ar = A.view(m, K2)
        Ar[0].zero_(); Ar[0, out] = 2.0
        Ar[1, out] = float("nan")
        Ar[2:20] /= torch.linalg.vector_norm(Ar[2:20], dim=1, keepdim=True)
    if opB == 0:  # B k-major
        Br = B.view(n, K2)
        Br[0].zero_(); Br[0, out] = -3.0
        Br[1, out + 1] = float("inf")
        Br[2:20] /= torch.linalg.vector_norm(Br[2:20], dim=1, keepdim=True)
    C0 = torch.rand(r * m * n, dtype=rt, device="cuda", generator=g) * 2 - 1
    alpha, beta = ((0.5 - 0.25j), (1.0 + 0.5j)) if cplx else (0.5, -1.0)
    ws_bytes = spla.splab_gemm_workspace_size(dt, spla.PATH_OZAKI, opA, opB, m, n, k)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    L = spla.lib()
    nphase = 20
    st = torch.cuda.Stream()
    outs, ran = [], []
    for onepass in ("1", "0"):
        os.environ["SPLAB_OZAKI_ONEPASS"] = onepass
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * nphase)]
        for e in ev:
            e.record(st)
        st.synchronize()
        handles = (ct.c_void_p * (2 * nphase))(*[e.cuda_event for e in ev])
        C = C0.clone()
        torch.cuda.synchronize()
        L.splab_set_phase_events(handles, nphase)
        try:
            rc = spla.splab_gemm(dt, spla.PATH_OZAKI, opA, opB, m, n, k, alpha, A, lda, B, ldb,
                                 beta, C, m, workspace=ws, workspace_bytes=ws_bytes,
                                 stream=st.cuda_stream)
        finally:
            L.splab_set_phase_events(None, 0)
            os.environ.pop("SPLAB_OZAKI_ONEPASS", None)
        assert rc == 0
        st.synchronize()
        outs.append(C.cpu().numpy())
        ran.append(ev[37].elapsed_time(ev[39]) if onepass == "1" else ev[39].elapsed_time(ev[37]))
    assert ran[0] > 0.0 and ran[1] > 0.0, ran
    assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8))
    Rdt = torch.complex128 if cplx else torch.float64
    R = torch.zeros(m * n, dtype=Rdt, device="cuda")
    Ad, Bd = A.double(), B.double()
    if cplx:
        Ad, Bd = torch.view_as_complex(Ad.view(-1, 2)), torch.view_as_complex(Bd.view(-1, 2))
    assert spla.gemm_dd("complex128" if cplx else "float64", opA, opB, m, n, k, Ad, lda, Bd, ldb,
                        R, m) == 0
    torch.cuda.synchronize()
    c0 = C0.double().cpu().numpy()
    got = outs[0].astype(np.float64)
    if cplx:
        got, c0 = got.view(np.complex128), c0.view(np.complex128)
    ref = alpha * R.cpu().numpy() + beta * c0
    bad = np.zeros((n, m), bool)  # column-major C: [column][row]
    if opA != 0:
        bad[:, 1] = True
    if opB == 0:
        bad[1, :] = True
    got, ref, bad = got.reshape(n, m), ref.reshape(n, m), bad
    assert np.isnan(got[bad]).all()
    tol = 1e-14 if rt == torch.float64 else 1e-6
    ok = ~bad
    assert oracle.rel_fro(got[ok], ref[ok]) <= tol
