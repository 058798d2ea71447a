"""GPU parity: libspla.so (sm_100a kernels) through the spla_* C ABI against the
golden outputs of the reference library on the same seeded inputs.

Checks per case: computed elements within tolerance of the reference's result
(golden_cases.tolerance), every element of the C buffer outside the m x n
block bit-unchanged (exact C layout, ldc padding untouched), and for
pgemm_ssbtr every element either the reference's value or unchanged.
Operands are passed as device pointers and, for a subset, as host pointers
(the streamed path). Every case runs on the automatic path choice and with
each contraction path forced (FP64 DMMA, Ozaki INT8, 3xTF32), so the
reference's own outputs pin the tensor-core paths directly; a forced path
that does not support a case (3xTF32 on double dtypes) runs DMMA, and each
test checks that the forced path took some of its cases."""
import ctypes as ct
import json

import numpy as np
import pytest

import golden_cases as gc
from capi import SplaCAPI

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ours(spla_lib):
    return SplaCAPI(spla_lib.LIB_PATH)


PATHS = {0: "auto", 1: "dmma", 2: "ozaki", 3: "tf32x3"}


@pytest.fixture(scope="module", params=list(PATHS), ids=list(PATHS.values()))
def ctx(ours, request):
    h = ours.ctx(1)
    ours.lib.spla_b200_ctx_set_fp64_path.argtypes = [ct.c_void_p, ct.c_int, ct.c_int]
    assert ours.lib.spla_b200_ctx_set_fp64_path(h, request.param, 0) == 0
    h.path = request.param
    yield h
    ours.destroy_ctx(h)


class PathCount:
    """How many cases the forced path itself computed (splab_gemm_path)."""

    def __init__(self, lib, ctx):
        self.lib, self.path, self.taken, self.total = lib, ctx.path, 0, 0
        lib.splab_gemm_path.argtypes = [ct.c_int] * 4 + [ct.c_int64] * 3
        lib.splab_gemm_path.restype = ct.c_int

    def add(self, dt, opA, opB, m, n, k):
        self.total += 1
        code = {np.float32: 0, np.float64: 1, np.complex64: 2, np.complex128: 3}[dt]
        if self.path and self.lib.splab_gemm_path(code, self.path, opA, opB, m, n, k) == self.path:
            self.taken += 1

    def check(self, expect_taken=True):
        if self.path in (2, 3) and expect_taken:
            assert self.taken > 0, f"path {self.path} took none of {self.total} cases"


def dev(x):
    import torch
    return torch.from_numpy(x).cuda() if x is not None else None


def host(t):
    return t.cpu().numpy()


def bound(c, dt, A, B, C0):
    alpha = abs(gc.scalar(c["alpha"], dt))
    beta = abs(gc.scalar(c["beta"], dt))
    amax = np.abs(A).max() if A.size else 0.0
    bmax = np.abs(B).max() if B.size else 0.0
    return alpha * max(1, c["k"]) * amax * bmax * 2 + beta * (np.abs(C0).max() if C0.size else 0)


def check_case(name, c, dt, A, B, C0, Cout, mask_fn=None):
    idx, val = gc.expected(name, c)
    tol = gc.tolerance(dt, c["k"]) * bound(c, dt, A, B, C0)
    got = Cout[idx]
    if mask_fn is None:
        err = np.abs(got - val).max() if idx.size else 0.0
        assert err <= tol, (name, c, err, tol)
        return
    inside, tri = mask_fn(idx)
    # outside the block: bit-identical to the input
    assert np.array_equal(got[~inside], C0[idx][~inside]), (name, c, "outside block changed")
    # in the triangle: the reference's value
    if tri.any():
        err = np.abs(got[tri] - val[tri]).max()
        assert err <= tol, (name, c, err, tol)
    # in the block but outside the triangle: either computed or untouched
    rest = inside & ~tri
    if rest.any():
        ok = (np.abs(got[rest] - val[rest]) <= tol) | (got[rest] == C0[idx][rest])
        assert ok.all(), (name, c, "off-triangle element neither computed nor unchanged")


@pytest.mark.parametrize("use_host", [False, True])
def test_gemm_grid(ours, ctx, use_host):
    cases, _ = gc.load("gemm")
    sel = cases if not use_host else cases[::5]
    count = PathCount(ours.lib, ctx)
    for c in sel:
        dt, A, B, C = gc.gemm_inputs(c)
        count.add(dt, c["opA"], c["opB"], c["m"], c["n"], c["k"])
        C0 = C.copy()
        if use_host:
            rc = ours.gemm(dt, c["opA"], c["opB"], c["m"], c["n"], c["k"], c["alpha"], A, c["lda"],
                           B, c["ldb"], c["beta"], C, c["ldc"], ctx)
            out = C
        else:
            dA, dB, dC = dev(A), dev(B), dev(C)
            rc = ours.gemm(dt, c["opA"], c["opB"], c["m"], c["n"], c["k"], c["alpha"], dA,
                           c["lda"], dB, c["ldb"], c["beta"], dC, c["ldc"], ctx)
            out = host(dC)
        assert rc == 0, (c, rc)
        check_case("gemm", c, dt, A, B, C0, out,
                   mask_fn=lambda idx, c=c: (_block_mask(c, idx), _block_mask(c, idx)))
    count.check()


def _block_mask(c, idx):
    ldc = c["ldc"]
    r, col = idx % ldc, idx // ldc
    return (r < c["m"]) & (col < c["n"])


@pytest.mark.parametrize("use_host", [False, True])
def test_ssb_and_ssbtr(ours, ctx, use_host):
    cases, _ = gc.load("ssb")
    sel = cases if not use_host else cases[::4]
    count = PathCount(ours.lib, ctx)
    for c in sel:
        dt, A, B, C = gc.ssb_inputs(c)
        count.add(dt, c["opA"], 0, c["m"], c["n"], c["k"])
        C0 = C.copy()
        rcd, dist = ours.block_cyclic(1, 1, 64, 64)
        alpha, beta = gc.scalar(c["alpha"], dt), gc.scalar(c["beta"], dt)
        if use_host:
            rc = ours.pgemm_ssbtr(dt, c["m"], c["n"], c["k"], c["opA"], alpha, A, c["lda"], B,
                                  c["ldb"], beta, C, c["ldc"], c["ro"], c["co"], c["fill"], dist,
                                  ctx)
            out = C
        else:
            dA, dB, dC = dev(A), dev(B), dev(C)
            rc = ours.pgemm_ssbtr(dt, c["m"], c["n"], c["k"], c["opA"], alpha, dA, c["lda"], dB,
                                  c["ldb"], beta, dC, c["ldc"], c["ro"], c["co"], c["fill"], dist,
                                  ctx)
            out = host(dC)
        assert rc == 0, (c, rc)

        def masks(idx, c=c):
            inside = gc.fill_mask({**c, "fill": 0}, idx)
            return inside, gc.fill_mask(c, idx)

        check_case("ssb", c, dt, A, B, C0, out, mask_fn=masks)
    count.check()


@pytest.mark.parametrize("use_host", [False, True])
def test_sbs(ours, ctx, use_host):
    cases, _ = gc.load("sbs")
    sel = cases if not use_host else cases[::3]
    count = PathCount(ours.lib, ctx)
    for c in sel:
        dt, A, B, C = gc.sbs_inputs(c)
        count.add(dt, 0, 0, c["mloc"], c["n"], c["k"])
        C0 = C.copy()
        rcd, dist = ours.block_cyclic(1, 1, 128, 128)
        alpha, beta = gc.scalar(c["alpha"], dt), gc.scalar(c["beta"], dt)
        if use_host:
            rc = ours.pgemm_sbs(dt, c["mloc"], c["n"], c["k"], alpha, A, c["lda"], B, c["ldb"],
                                c["bro"], c["bco"], dist, beta, C, c["ldc"], ctx)
            out = C
        else:
            dA, dB, dC = dev(A), dev(B), dev(C)
            rc = ours.pgemm_sbs(dt, c["mloc"], c["n"], c["k"], alpha, dA, c["lda"], dB, c["ldb"],
                                c["bro"], c["bco"], dist, beta, dC, c["ldc"], ctx)
            out = host(dC)
        assert rc == 0, (c, rc)

        def masks(idx, c=c):
            r, col = idx % c["ldc"], idx // c["ldc"]
            inside = (r < c["mloc"]) & (col < c["n"])
            return inside, inside

        check_case("sbs", c, dt, A, B, C0, out, mask_fn=masks)
    count.check(expect_taken=ctx.path == 2)  # 3xTF32 takes op(A) in {T, C} only


def test_error_codes(ours, ctx):
    """Invalid calls return the reference's codes (errors.json). Documented
    divergence: ldc < m is rejected (SPLA_INVALID_PARAMETER_ERROR) where the
    reference hands it to BLAS, which refuses to compute."""
    cases = json.loads((gc.GOLDEN / "errors.json").read_text())
    rcd, dist = ours.block_cyclic(1, 1, 64, 64)
    A = dev(np.ones(1000))
    for c in cases:
        a = c["args"]
        C = dev(np.ones(1000))
        p = lambda key: A if a.get(key, 1) else None  # noqa: E731
        cp = C if a.get("C", 1) else None
        d = np.float64
        if c["call"] == "ssb":
            rc = ours.pgemm_ssb(d, a["m"], a["n"], a["k"], a["opA"], 1.0, p("A"), a["lda"], p("B"),
                                a["ldb"], 0.0, cp, a["ldc"], a["ro"], a["co"], dist, ctx)
        elif c["call"] == "sbs":
            rc = ours.pgemm_sbs(d, a["m"], a["n"], a["k"], 1.0, p("A"), a["lda"], p("B"), a["ldb"],
                                a["bro"], a["bco"], dist, 0.0, cp, a["ldc"], ctx)
        else:
            rc = ours.gemm(d, a["opA"], a["opB"], a["m"], a["n"], a["k"], 1.0, p("A"), a["lda"],
                           p("B"), a["ldb"], 0.0, cp, a["ldc"], ctx)
        expect = 3 if c["name"] == "gemm ldc small is accepted" else c["code"]
        assert rc == expect, c


def test_cfg1_full(ours, ctx):
    """pdgemm_ssb k=20000, m=n=256, op=T, U[-1,1]: full C vs the reference."""
    from inputs import buffer
    import oracle
    g = np.load(gc.GOLDEN / "cfg1.npz")
    k, m, n = int(g["k"]), int(g["m"]), int(g["n"])
    A = buffer(np.float64, k, m, 20250001, "uniform11")
    B = buffer(np.float64, k, n, 20250002, "uniform11")
    dC = dev(np.zeros(m * n))
    rcd, dist = ours.block_cyclic(1, 1, 64, 64)
    rc = ours.pgemm_ssb(np.float64, m, n, k, 1, 1.0, dev(A), k, dev(B), k, 0.0, dC, m, 0, 0, dist,
                        ctx)
    assert rc == 0
    assert oracle.rel_fro(host(dC), g["C"]) < 1e-14


@pytest.mark.parametrize("dtn,opA", [("z", 2), ("d", 1), ("c", 2), ("s", 1)])
def test_ssb_streamed_host_operands(dtn, opA):
    """Host-resident A and B streamed in many k-chunks (tile_size_gpu forced
    small): the chunked accumulation (beta on the first chunk, 1 after) equals
    the oracle on the same inputs."""
    import spla_b200 as spla
    import oracle
    from inputs import buffer
    dt = gc.DT[dtn]
    m, n, k = 70, 45, 5003
    A = buffer(dt, k + 1, m, 101, "uniform11")
    B = buffer(dt, k + 2, n, 102, "uniform11")
    C = buffer(dt, m + 3, n, 103, "uniform11")
    ref = C.copy()
    alpha, beta = (0.5 + 0.25j, -1.0 + 0.5j) if dtn in "cz" else (0.5, -1.0)
    assert oracle.pgemm_ssb(m, n, k, opA, alpha, A, k + 1, B, k + 2, beta, ref, m + 3, 0, 0) == 0
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_tile_size_gpu(64)
    dist = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 64, 64)
    spla.pgemm_ssb(m, n, k, opA, alpha, A, k + 1, B, k + 2, beta, C, m + 3, 0, 0, dist, ctx)
    tol = 1e-6 if dtn in "sc" else 1e-14
    assert oracle.rel_fro(C, ref) <= tol
