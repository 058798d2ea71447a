"""Accuracy at the benchmark's scale of k against the double-double (Dot2)
oracle, through the spla_* C ABI with device-resident operands.

Bars: relative Frobenius error <= 1e-14 for double and
complex double; <= 1e-6 against the reference (so <= 5e-7 against the exact
result) for float."""
import numpy as np
import pytest

import oracle
from capi import SplaCAPI
from inputs import buffer

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ours(spla_lib):
    return SplaCAPI(spla_lib.LIB_PATH)


def _dev(x):
    import torch
    return torch.from_numpy(x).cuda()


def _oracle_ssb(dt, m, n, k, opA, A, B):
    C = np.zeros(m * n, dt)
    assert oracle.pgemm_ssb(m, n, k, opA, 1.0, A, k, B, k, 0.0, C, m, 0, 0) == 0
    return C


@pytest.mark.parametrize("path", [1, 2], ids=["dmma", "ozaki"])
def test_zgemm_ssb_k250000(ours, path):
    import spla_b200
    m = n = 48
    k = 250000
    dt = np.complex128
    A = buffer(dt, k, m, 11, "gauss_k", k)
    B = buffer(dt, k, n, 12, "gauss_k", k)
    ctx = spla_b200.Context(spla_b200.PU_GPU)
    ctx.set_fp64_path(path)
    rc, dist = ours.block_cyclic(1, 1, 128, 128)
    dC = _dev(np.zeros(m * n, dt))
    rc = ours.pgemm_ssb(dt, m, n, k, 2, 1.0, _dev(A), k, _dev(B), k, 0.0, dC, m, 0, 0, dist,
                        ctx.handle)
    assert rc == 0
    err = oracle.rel_fro(dC.cpu().numpy(), _oracle_ssb(dt, m, n, k, 2, A, B))
    assert err <= 1e-14, err


def test_dgemm_ssb_k100000(ours):
    import spla_b200
    m, n, k = 40, 72, 100000
    dt = np.float64
    A = buffer(dt, k, m, 21, "uniform11")
    B = buffer(dt, k, n, 22, "uniform11")
    ctx = spla_b200.Context(spla_b200.PU_GPU)
    rc, dist = ours.block_cyclic(1, 1, 64, 64)
    dC = _dev(np.zeros(m * n, dt))
    assert ours.pgemm_ssb(dt, m, n, k, 1, 1.0, _dev(A), k, _dev(B), k, 0.0, dC, m, 0, 0, dist,
                          ctx.handle) == 0
    err = oracle.rel_fro(dC.cpu().numpy(), _oracle_ssb(dt, m, n, k, 1, A, B))
    assert err <= 1e-14, err


@pytest.mark.parametrize("path", [1, 2, 3], ids=["dmma", "ozaki", "tf32x3"])
def test_sgemm_ssbtr_lower_k400000(ours, path):
    """Real float ssbtr, fill LOWER, k = 400000 (the triangle is checked), on
    each path."""
    import spla_b200
    m = n = 64
    k = 400000
    dt = np.float32
    A = buffer(dt, k, m, 31, "gauss_k", k)
    B = buffer(dt, k, n, 32, "gauss_k", k)
    ctx = spla_b200.Context(spla_b200.PU_GPU)
    ctx.set_fp64_path(path)
    rc, dist = ours.block_cyclic(1, 1, 64, 64)
    dC = _dev(np.zeros(m * n, dt))
    assert ours.pgemm_ssbtr(dt, m, n, k, 1, 1.0, _dev(A), k, _dev(B), k, 0.0, dC, m, 0, 0, 2,
                            dist, ctx.handle) == 0
    ref = np.zeros(m * n, np.float64)
    assert oracle.gemm(1, 0, m, n, k, 1.0, A.astype(np.float64), k, B.astype(np.float64), k, 0.0,
                       ref, m) == 0
    got = dC.cpu().numpy().reshape(n, m).T.astype(np.float64)
    ex = ref.reshape(n, m).T
    tri = np.tril(np.ones((m, n), bool))
    err = np.linalg.norm((got - ex)[tri]) / np.linalg.norm(ex[tri])
    assert err <= 5e-7, err


@pytest.mark.parametrize("use_host", [False, True], ids=["device", "pinned_host"])
def test_zgemm_ssb_ozaki_k250000_whole_c(ours, use_host):
    """The headline contraction (A^H B, complex double, k = 250000) on the
    Ozaki path with m = n = 256, the whole C checked against the device
    double-double reference (itself pinned to the CPU Dot2 oracle on three
    columns here); operands in device memory and in pinned host memory
    (streamed in k-chunks through the public C ABI)."""
    import torch
    import spla_b200
    m = n = 256
    k = 250000
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    s = (1.0 / (2.0 * k)) ** 0.5
    A = torch.randn((m, k), dtype=torch.complex128, device="cuda", generator=g) * s
    B = torch.randn((n, k), dtype=torch.complex128, device="cuda", generator=g) * s
    R = torch.zeros((n, m), dtype=torch.complex128, device="cuda")
    assert spla_b200.gemm_dd(3, 2, 0, m, n, k, A, k, B, k, R, m) == 0
    torch.cuda.synchronize()
    cols = [0, 129, 255]
    ref = np.zeros(m * len(cols), np.complex128)
    An = A.cpu().numpy().ravel()
    assert oracle.gemm(2, 0, m, len(cols), k, 1.0, An, k,
                       np.ascontiguousarray(B[cols].cpu().numpy().ravel()), k, 0.0, ref, m) == 0
    assert oracle.rel_fro(R[cols].cpu().numpy().ravel(), ref) <= 1e-16
    ctx = spla_b200.Context(spla_b200.PU_GPU)
    ctx.set_fp64_path(spla_b200.PATH_OZAKI)
    dist = spla_b200.MatrixDistribution.create_blacs_block_cyclic(spla_b200.MPI_COMM_SELF, "R",
                                                                  1, 1, 128, 128)
    if use_host:
        hA, hB = A.cpu().pin_memory(), B.cpu().pin_memory()
        C = torch.zeros((n, m), dtype=torch.complex128).pin_memory()
        spla_b200.pgemm_ssb(m, n, k, 2, 1.0, hA, k, hB, k, 0.0, C, m, 0, 0, dist, ctx)
    else:
        C = torch.zeros((n, m), dtype=torch.complex128, device="cuda")
        spla_b200.pgemm_ssb(m, n, k, 2, 1.0, A, k, B, k, 0.0, C, m, 0, 0, dist, ctx)
        torch.cuda.synchronize()
    err = float(torch.linalg.vector_norm(C.cuda() - R) / torch.linalg.vector_norm(R))
    assert err <= 1e-14, err
