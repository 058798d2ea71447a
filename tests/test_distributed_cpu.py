"""Multi-rank pgemm_ssb / pgemm_sbs (spla_b200.distributed) on gloo ranks, CPU.

Each rank is a process of a world of 2 or 4 over gloo (127.0.0.1). The
exchange plans come from the library's host code (the reference's
block-cyclic map), the collectives are real gloo collectives, and the local
products and block moves run on a host backend (the compensated oracle and
numpy) because this machine has no GPU; the device kernels of the same steps
are checked on one GPU in tests/test_gpu_distributed.py.

Every rank's result is compared with the reference library's single-rank
result on the whole problem (the stripes of all ranks stacked along k, or the
whole B), laid out in the rank's local block-cyclic layout: elements outside
the submatrix stay unchanged, and fill modes are checked on the triangle.
Also: the owners of a grid reordered by a mapping, excess ranks outside the
grid, a mirror C, the reference's validation order and its local-size rule,
which the reference library answers for the same arguments."""
import ctypes as ct
import os
import socket

import numpy as np
import pytest

import oracle

REF = oracle.REF_LIB


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def numroc(n, nb, p, nprocs):
    """Rows of a dimension of n in blocks of nb held by grid coordinate p (ScaLAPACK)."""
    nblocks = n // nb
    num = (nblocks // nprocs) * nb
    extra = nblocks % nprocs
    if p < extra:
        num += nb
    elif p == extra:
        num += n % nb
    return num


class HostBackend:
    """Local products with the compensated oracle, block moves with numpy."""

    def empty(self, like, count):
        import torch
        return torch.zeros(max(1, count), dtype=like.dtype)

    def product(self, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        An = None if A is None else A.numpy()
        Bn = None if B is None else B.numpy()
        rc = oracle.gemm(opA, opB, m, n, k, alpha, An, lda, Bn, ldb, beta, C.numpy(), ldc)
        assert rc == 0, rc

    def copy_blocks(self, src, dst, desc, alpha, beta):
        s, d = src.numpy(), dst.numpy()
        for so, sld, do, dld, r, c in np.asarray(desc).reshape(-1, 6):
            for j in range(c):
                col = alpha * s[so + j * sld:so + j * sld + r]
                if beta != 0:
                    col = col + beta * d[do + j * dld:do + j * dld + r]
                d[do + j * dld:do + j * dld + r] = col


def _global_to_local(dist, gi, gj):
    R, C = dist.proc_grid_rows, dist.proc_grid_cols
    rb, cb = dist.row_block_size, dist.col_block_size
    g = (gi // rb) % R + ((gj // cb) % C) * R
    return dist.full_mapping[g], (gi // (rb * R)) * rb + gi % rb, (gj // (cb * C)) * cb + gj % cb


def _mat(buf, ld, rows, cols):
    return buf[:ld * cols].reshape(cols, ld)[:, :rows].T


def _ssb_case(rank, world, case):
    import torch
    import torch.distributed as tdist
    import spla_b200.distributed as sd
    from capi import SplaCAPI
    from inputs import buffer
    dt = case["dtype"]
    m, n, ro, co = case["m"], case["n"], case["ro"], case["co"]
    opA, fill = case["opA"], case.get("fill", 0)
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, 1.5)
    rng = np.random.default_rng(42)  # all ranks draw the same k splits
    ks = [int(x) for x in rng.integers(0, 400, world)]
    if case.get("zero_k_rank") is not None:
        ks[case["zero_k_rank"]] = 0
    K = sum(ks)
    A = buffer(dt, max(K, 1), m, 7, "uniform11")
    B = buffer(dt, max(K, 1), n, 8, "uniform11")
    grows, gcols = ro + m, co + n
    Cg = buffer(dt, grows, gcols, 9, "uniform11")
    # the reference's single-rank result on the stacked stripes
    ref = SplaCAPI(REF)
    h = ref.ctx(0)
    _, d1 = ref.block_cyclic(1, 1, 64, 64)
    expect = Cg.copy()
    assert ref.pgemm_ssbtr(dt, m, n, K, opA, alpha, A, max(K, 1), B, max(K, 1), beta, expect,
                           grows, ro, co, fill, d1, h) == 0
    # this rank's stripe
    k0 = sum(ks[:rank])
    kl = ks[rank]
    Am = _mat(A, max(K, 1), K, m)[k0:k0 + kl]
    Bm = _mat(B, max(K, 1), K, n)[k0:k0 + kl]
    lda = kl + 2
    Al = np.zeros(lda * m, dt)
    Bl = np.zeros(lda * n, dt)
    _mat(Al, lda, kl, m)[:] = Am
    _mat(Bl, lda, kl, n)[:] = Bm
    if case["dist"] == "mirror":
        dist = sd.Distribution.create_mirror(None)
        Cl = Cg.copy()
        ldc = grows
        sd.pgemm_ssb(m, n, kl, opA, alpha, torch.from_numpy(Al), lda, torch.from_numpy(Bl), lda,
                     beta, torch.from_numpy(Cl), ldc, ro, co, dist, HostBackend(), fill)
        got = Cl
        want = expect
    else:
        R, Cc, rb, cb = case["grid"]
        if case.get("mapping") is not None:
            dist = sd.Distribution.create_blacs_block_cyclic_from_mapping(None, case["mapping"],
                                                                          R, Cc, rb, cb)
        else:
            dist = sd.Distribution.create_blacs_block_cyclic(None, case.get("order", "R"), R,
                                                             Cc, rb, cb)
        g = dist.grid_index(rank)
        pr, pc = (g % R, g // R) if g < R * Cc else (None, None)
        lr = numroc(grows, rb, pr, R) if pr is not None else 0
        lc = numroc(gcols, cb, pc, Cc) if pc is not None else 0
        ldc = lr + 3
        Cl = buffer(dt, ldc, max(lc, 1), 100 + rank, "uniform11")
        # local C starts as the distributed global C (padding keeps its own data)
        want = Cl.copy()
        for gj in range(gcols):
            for gi in range(grows):
                p, li, lj = _global_to_local(dist, gi, gj)
                if p == rank:
                    Cl[li + lj * ldc] = Cg[gi + gj * grows]
                    want[li + lj * ldc] = expect[gi + gj * grows]
        before = Cl.copy()
        sd.pgemm_ssb(m, n, kl, opA, alpha, torch.from_numpy(Al), lda, torch.from_numpy(Bl), lda,
                     beta, torch.from_numpy(Cl), ldc, ro, co, dist, HostBackend(), fill)
        got = Cl
        if fill:
            # off the triangle an element is either computed or unchanged
            for gj in range(gcols):
                for gi in range(grows):
                    p, li, lj = _global_to_local(dist, gi, gj)
                    tri = gi >= gj if fill == 2 else gj >= gi
                    x = li + lj * ldc
                    if p == rank and not tri and got[x] == before[x]:
                        want[x] = before[x]
    tol = 1e-12 if np.dtype(dt) in (np.float64, np.complex128) else 1e-5
    scale = max(1.0, np.abs(want).max())
    assert np.allclose(got, want, rtol=0, atol=tol * scale * max(K, 1) / 100), (
        rank, np.abs(got - want).max())
    tdist.barrier()


def _sbs_case(rank, world, case):
    import torch
    import torch.distributed as tdist
    import spla_b200.distributed as sd
    from capi import SplaCAPI
    from inputs import buffer
    dt = case["dtype"]
    k, n, bro, bco = case["k"], case["n"], case["bro"], case["bco"]
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = (0.75 + 0.5j, -0.5 + 1.0j) if cplx else (0.75, -0.5)
    rng = np.random.default_rng(43)
    ms = [int(x) for x in rng.integers(1, 60, world)]
    ml = ms[rank]
    grows, gcols = bro + k, bco + n
    Bg = buffer(dt, grows, gcols, 11, "uniform11")
    A = buffer(dt, ml + 1, k, 20 + rank, "uniform11")
    C = buffer(dt, ml + 2, n, 30 + rank, "uniform11")
    ref = SplaCAPI(REF)
    h = ref.ctx(0)
    _, d1 = ref.block_cyclic(1, 1, 64, 64)
    want = C.copy()
    assert ref.pgemm_sbs(dt, ml, n, k, alpha, A, ml + 1, Bg, grows, bro, bco, d1, beta, want,
                         ml + 2, h) == 0
    R, Cc, rb, cb = case["grid"]
    if case.get("mapping") is not None:
        dist = sd.Distribution.create_blacs_block_cyclic_from_mapping(None, case["mapping"], R,
                                                                      Cc, rb, cb)
    else:
        dist = sd.Distribution.create_blacs_block_cyclic(None, "R", R, Cc, rb, cb)
    g = dist.grid_index(rank)
    pr, pc = (g % R, g // R) if g < R * Cc else (None, None)
    lr = numroc(grows, rb, pr, R) if pr is not None else 0
    lc = numroc(gcols, cb, pc, Cc) if pc is not None else 0
    ldb = max(lr, 1) + 1
    Bl = np.zeros(ldb * max(lc, 1), dt)
    for gj in range(gcols):
        for gi in range(grows):
            p, li, lj = _global_to_local(dist, gi, gj)
            if p == rank:
                Bl[li + lj * ldb] = Bg[gi + gj * grows]
    got = C.copy()
    sd.pgemm_sbs(ml, n, k, alpha, torch.from_numpy(A), ml + 1, torch.from_numpy(Bl), ldb, bro,
                 bco, dist, beta, torch.from_numpy(got), ml + 2, HostBackend())
    tol = 1e-12 if np.dtype(dt) in (np.float64, np.complex128) else 1e-5
    scale = max(1.0, np.abs(want).max())
    assert np.allclose(got, want, rtol=0, atol=tol * scale * k / 50), (rank,
                                                                       np.abs(got - want).max())
    tdist.barrier()


def _errors_case(rank, world, case):
    import torch
    import torch.distributed as tdist
    import spla_b200 as spla
    import spla_b200.distributed as sd
    d = sd.Distribution.create_blacs_block_cyclic(None, "R", 1, world, 4, 4)
    x = torch.zeros(256, dtype=torch.float64)
    with pytest.raises(spla.InvalidParameterError):  # op(A) = N
        sd.pgemm_ssb(8, 8, 4, spla.OP_NONE, 1.0, x, 4, x, 4, 0.0, x, 8, 0, 0, d, HostBackend())
    with pytest.raises(spla.InvalidParameterError):  # negative offset
        sd.pgemm_ssb(8, 8, 4, spla.OP_TRANSPOSE, 1.0, x, 4, x, 4, 0.0, x, 8, -1, 0, d,
                     HostBackend())
    # m = 0 returns before checking op(A), as the reference
    sd.pgemm_ssb(0, 8, 4, spla.OP_NONE, 1.0, x, 4, x, 4, 0.0, x, 8, 0, 0, d, HostBackend())
    with pytest.raises(spla.InvalidParameterError):  # lda < kLocal
        sd.pgemm_ssb(8, 8, 8, spla.OP_TRANSPOSE, 1.0, x, 4, x, 8, 0.0, x, 8, 0, 0, d,
                     HostBackend())
    with pytest.raises(spla.InvalidPointerError):  # null B with kLocal > 0 (4 local columns)
        sd.pgemm_ssb(8, 8, 4, spla.OP_TRANSPOSE, 1.0, x, 4, None, 4, 0.0, x, 8, 0, 0, d,
                     HostBackend())
    with pytest.raises(spla.InvalidParameterError):  # mapping: repeated rank
        sd.Distribution.create_blacs_block_cyclic_from_mapping(None, [0] * world, 1, world, 4, 4)
    with pytest.raises(spla.InvalidParameterError):  # grid larger than the group
        sd.Distribution.create_blacs_block_cyclic(None, "R", world + 1, 1, 4, 4)
    with pytest.raises(spla.InvalidParameterError):  # order
        sd.Distribution.create_blacs_block_cyclic(None, "X", 1, 1, 4, 4)
    # sbs: k = 0 returns before any check; negative offsets on a block-cyclic B
    sd.pgemm_sbs(4, 4, 0, 1.0, None, 4, None, 4, -1, 0, d, 0.0, x, 4, HostBackend())
    with pytest.raises(spla.InvalidParameterError):
        sd.pgemm_sbs(4, 4, 4, 1.0, x, 4, x, 4, -1, 0, d, 0.0, x, 4, HostBackend())
    tdist.barrier()


def _local_size_case(rank, world, case):
    """Distribution.local_size equals the reference generator's local_rows /
    local_cols (block_cyclic_generator.cpp:117-141), including its rule for a
    partial last block, for grids, offsets and block sizes."""
    import torch.distributed as tdist
    import spla_b200.distributed as sd
    L = ct.CDLL(str(REF))
    for f in (L.ref_local_rows, L.ref_local_cols):
        f.argtypes = [ct.c_long] * 9
        f.restype = ct.c_long
    rng = np.random.default_rng(5 + rank)
    for _ in range(300):
        R, Cc = int(rng.integers(1, 4)), int(rng.integers(1, 4))
        rb, cb = int(rng.integers(1, 9)), int(rng.integers(1, 9))
        nr, nc = int(rng.integers(0, 40)), int(rng.integers(0, 40))
        ro, co = int(rng.integers(0, 12)), int(rng.integers(0, 12))
        d = sd.Distribution(0, None, R, Cc, rb, cb, list(range(R * Cc)))
        for g in range(R * Cc):
            got = d.local_size(nr, nc, ro, co, g)
            want = (L.ref_local_rows(rb, cb, R, Cc, nr, nc, ro, co, g),
                    L.ref_local_cols(rb, cb, R, Cc, nr, nc, ro, co, g))
            assert got == want, (R, Cc, rb, cb, nr, nc, ro, co, g, got, want)
    tdist.barrier()


def _run(rank, world, port, fn_name, case):
    import torch.distributed as tdist
    import datetime
    tdist.init_process_group("gloo", rank=rank, world_size=world,
                             init_method=f"tcp://127.0.0.1:{port}",
                             timeout=datetime.timedelta(seconds=120))
    try:
        globals()[fn_name](rank, world, case)  # distributions on the default group
    finally:
        tdist.destroy_process_group()


def _spawn(fn_name, case, world=2):
    import torch.multiprocessing as mp
    if not REF.exists():
        pytest.skip("reference library not built (oracle/_ref)")
    mp.spawn(_run, args=(world, _port(), fn_name, case), nprocs=world, join=True)


SSB_CASES = [
    dict(dtype=np.float64, m=13, n=9, ro=2, co=3, opA=1, dist="bc", grid=(2, 1, 3, 5)),
    dict(dtype=np.complex128, m=21, n=17, ro=0, co=4, opA=2, dist="bc", grid=(1, 2, 4, 3)),
    dict(dtype=np.complex128, m=21, n=17, ro=1, co=1, opA=2, dist="bc", grid=(1, 2, 4, 3),
         mapping=[1, 0]),
    dict(dtype=np.float32, m=32, n=32, ro=0, co=0, opA=1, dist="bc", grid=(2, 1, 8, 8),
         order="C"),
    dict(dtype=np.complex64, m=19, n=19, ro=3, co=2, opA=2, dist="bc", grid=(1, 2, 5, 5),
         fill=2),
    dict(dtype=np.float64, m=15, n=15, ro=0, co=0, opA=1, dist="bc", grid=(2, 1, 4, 4), fill=1,
         zero_k_rank=1),
    dict(dtype=np.complex128, m=11, n=7, ro=2, co=1, opA=2, dist="mirror"),
]


@pytest.mark.parametrize("case", SSB_CASES, ids=[f"ssb{i}" for i in range(len(SSB_CASES))])
def test_ssb_two_ranks(case):
    _spawn("_ssb_case", case)


def test_ssb_four_ranks_2x2_grid():
    _spawn("_ssb_case", dict(dtype=np.complex128, m=23, n=18, ro=1, co=2, opA=2, dist="bc",
                             grid=(2, 2, 4, 3), mapping=[3, 1, 0, 2]), world=4)


def test_ssb_excess_rank_outside_grid():
    """Three ranks on a 1 x 2 grid: the third owns no block but takes part."""
    _spawn("_ssb_case", dict(dtype=np.float64, m=10, n=12, ro=0, co=1, opA=1, dist="bc",
                             grid=(1, 2, 3, 4), mapping=[2, 0]), world=3)


SBS_CASES = [
    dict(dtype=np.complex128, k=23, n=14, bro=2, bco=1, grid=(2, 1, 4, 3)),
    dict(dtype=np.float64, k=30, n=11, bro=0, bco=3, grid=(1, 2, 5, 4), mapping=[1, 0]),
    dict(dtype=np.complex64, k=17, n=20, bro=1, bco=0, grid=(2, 1, 3, 7)),
]


@pytest.mark.parametrize("case", SBS_CASES, ids=[f"sbs{i}" for i in range(len(SBS_CASES))])
def test_sbs_two_ranks(case):
    _spawn("_sbs_case", case)


def test_sbs_four_ranks_2x2_grid():
    _spawn("_sbs_case", dict(dtype=np.float64, k=29, n=19, bro=3, bco=2, grid=(2, 2, 4, 5)),
           world=4)


def test_validation_order_and_errors():
    _spawn("_errors_case", {})


def test_local_size_matches_reference():
    _spawn("_local_size_case", {})


def test_ssb_three_ranks_3x1_grid_with_mapping():
    """An odd rank count: a 3 x 1 grid whose grid indices map to ranks 1, 2, 0."""
    _spawn("_ssb_case", dict(dtype=np.complex64, m=17, n=13, ro=2, co=0, opA=2, dist="bc",
                             grid=(3, 1, 3, 4), mapping=[1, 2, 0]), world=3)


def test_sbs_three_ranks_1x3_grid_with_mapping():
    """B's blocks gathered from three ranks of a 1 x 3 grid mapped to ranks 2, 0, 1."""
    _spawn("_sbs_case", dict(dtype=np.complex128, k=31, n=16, bro=1, bco=2, grid=(1, 3, 4, 3),
                             mapping=[2, 0, 1]), world=3)
