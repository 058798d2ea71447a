"""Multi-rank pgemm_ssb / pgemm_sbs on the device kernels, one GPU.

The exchange steps of spla_b200.distributed run on the library's kernels
(local contraction, splab_copy_blocks) for every rank of a world emulated in
one process: each rank's partial product and packing run on the GPU, the
collective is replaced by its arithmetic (the sum of the ranks' send buffers
for the reduce-scatter, their concatenation for the all-gather), and each
rank's unpacking runs on the GPU. No kernel waits on another rank's. The
results are checked like the gloo tests (tests/test_distributed_cpu.py):
against the reference library's single-rank result laid out in each rank's
block-cyclic local C. The last test runs pgemm_ssb through a real NCCL
process group of one rank."""
import numpy as np
import pytest

import oracle
from test_distributed_cpu import _global_to_local, _mat, numroc

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("dt,opA,grid,mapping,ro,co,path", [
    (np.complex128, 2, (2, 2, 4, 3), [3, 1, 0, 2], 1, 2, 1),
    (np.complex128, 2, (1, 3, 8, 8), None, 0, 5, 2),
    (np.float64, 1, (2, 1, 5, 7), [1, 0], 3, 0, 2),
    (np.complex64, 2, (2, 2, 16, 16), None, 0, 0, 3),
])
def test_ssb_exchange_emulated(dt, opA, grid, mapping, ro, co, path):
    import torch
    import spla_b200 as spla
    import spla_b200.distributed as sd
    from capi import SplaCAPI
    from inputs import buffer
    if not oracle.REF_LIB.exists():
        pytest.skip("reference library not built (oracle/_ref)")
    R, Cc, rb, cb = grid
    world = R * Cc
    full = mapping or list(range(world))
    dist = sd.Distribution(spla.DIST_BLACS_BLOCK_CYCLIC, None, R, Cc, rb, cb, full)
    m, n = 45, 38
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, 1.5)
    ks = [int(x) for x in np.random.default_rng(3).integers(100, 3000, world)]
    K = sum(ks)
    A = buffer(dt, K, m, 7, "gauss_k", K)
    B = buffer(dt, K, n, 8, "gauss_k", K)
    grows, gcols = ro + m, co + n
    Cg = buffer(dt, grows, gcols, 9, "uniform11")
    ref = SplaCAPI(oracle.REF_LIB)
    _, d1 = ref.block_cyclic(1, 1, 64, 64)
    expect = Cg.copy()
    assert ref.pgemm_ssb(dt, m, n, K, opA, alpha, A, K, B, K, beta, expect, grows, ro, co, d1,
                         ref.ctx(0)) == 0
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    backend = sd.DeviceBackend(ctx)
    plan = sd.ssb_plan(dist, m, n, ro, co, 0)
    tdt = getattr(torch, np.dtype(dt).name)
    total = torch.zeros(world * plan.seg, dtype=tdt, device="cuda")
    k0 = 0
    for r in range(world):
        Al = np.ascontiguousarray(_mat(A, K, K, m)[k0:k0 + ks[r]].T).ravel()  # ks[r] x m, ld ks[r]
        Bl = np.ascontiguousarray(_mat(B, K, K, n)[k0:k0 + ks[r]].T).ravel()
        k0 += ks[r]
        P = backend.empty(total, m * n)
        backend.product(opA, 0, m, n, ks[r], 1.0, _dev(Al), ks[r], _dev(Bl), ks[r], 0.0, P, m)
        send = backend.empty(total, world * plan.seg)
        backend.copy_blocks(P, send, sd.ssb_pack_desc(plan, m), 1.0, 0.0)
        total += send  # the reduce-scatter's sums
    for r in range(world):
        g = dist.grid_index(r)
        lr, lc = numroc(grows, rb, g % R, R), numroc(gcols, cb, g // R, Cc)
        ldc = lr + 2
        Cl = buffer(dt, ldc, max(lc, 1), 50 + r, "uniform11")
        want = Cl.copy()
        for gj in range(gcols):
            for gi in range(grows):
                p, li, lj = _global_to_local(dist, gi, gj)
                if p == r:
                    Cl[li + lj * ldc] = Cg[gi + gj * grows]
                    want[li + lj * ldc] = expect[gi + gj * grows]
        dC = _dev(Cl)
        recv = total[r * plan.seg:(r + 1) * plan.seg].clone()
        backend.copy_blocks(recv, dC, sd.ssb_unpack_desc(plan, r, ldc), alpha, beta)
        torch.cuda.synchronize()
        got = dC.cpu().numpy()
        tol = 1e-13 if np.dtype(dt) in (np.float64, np.complex128) else 1e-5
        assert np.allclose(got, want, rtol=0, atol=tol * max(1.0, np.abs(want).max())), (
            r, np.abs(got - want).max())


@pytest.mark.parametrize("dt,grid,mapping,bro,bco,path", [
    (np.complex128, (2, 2, 4, 3), [2, 3, 0, 1], 2, 1, 1),
    (np.complex128, (2, 1, 64, 64), None, 0, 0, 2),
    (np.float32, (1, 2, 5, 4), [1, 0], 1, 3, 0),
])
def test_sbs_exchange_emulated(dt, grid, mapping, bro, bco, path):
    import torch
    import spla_b200 as spla
    import spla_b200.distributed as sd
    from capi import SplaCAPI
    from inputs import buffer
    if not oracle.REF_LIB.exists():
        pytest.skip("reference library not built (oracle/_ref)")
    R, Cc, rb, cb = grid
    world = R * Cc
    full = mapping or list(range(world))
    dist = sd.Distribution(spla.DIST_BLACS_BLOCK_CYCLIC, None, R, Cc, rb, cb, full)
    k, n = 150, 70
    cplx = np.dtype(dt).kind == "c"
    alpha, beta = (0.75 + 0.5j, -0.5 + 1.0j) if cplx else (0.75, -0.5)
    grows, gcols = bro + k, bco + n
    Bg = buffer(dt, grows, gcols, 11, "uniform11")
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(path)
    backend = sd.DeviceBackend(ctx)
    plan = sd.sbs_plan(dist, k, n, bro, bco)
    tdt = getattr(torch, np.dtype(dt).name)
    gathered = torch.zeros(world * plan.seg, dtype=tdt, device="cuda")
    for r in range(world):
        g = dist.grid_index(r)
        lr, lc = numroc(grows, rb, g % R, R), numroc(gcols, cb, g // R, Cc)
        ldb = max(lr, 1) + 1
        Bl = np.zeros(ldb * max(lc, 1), dt)
        for gj in range(gcols):
            for gi in range(grows):
                p, li, lj = _global_to_local(dist, gi, gj)
                if p == r:
                    Bl[li + lj * ldb] = Bg[gi + gj * grows]
        send = gathered[r * plan.seg:(r + 1) * plan.seg]  # the all-gather's layout
        backend.copy_blocks(_dev(Bl), send, sd.sbs_pack_desc(plan, r, ldb), 1.0, 0.0)
    Bfull = backend.empty(gathered, k * n)
    backend.copy_blocks(gathered, Bfull, sd.sbs_unpack_desc(plan, k), 1.0, 0.0)
    ref = SplaCAPI(oracle.REF_LIB)
    _, d1 = ref.block_cyclic(1, 1, 64, 64)
    for r in range(world):
        ml = 37 + 11 * r
        A = buffer(dt, ml, k, 20 + r, "uniform11")
        C = buffer(dt, ml + 1, n, 30 + r, "uniform11")
        want = C.copy()
        assert ref.pgemm_sbs(dt, ml, n, k, alpha, A, ml, Bg, grows, bro, bco, d1, beta, want,
                             ml + 1, ref.ctx(0)) == 0
        dC = _dev(C)
        backend.product(0, 0, ml, n, k, alpha, _dev(A), ml, Bfull, k, beta, dC, ml + 1)
        torch.cuda.synchronize()
        got = dC.cpu().numpy()
        tol = 1e-13 if np.dtype(dt) in (np.float64, np.complex128) else 1e-5
        assert np.allclose(got, want, rtol=0, atol=tol * k * max(1.0, np.abs(want).max())), (
            r, np.abs(got - want).max())


def test_ssb_through_nccl_one_rank():
    """pgemm_ssb of the distributed layer through a real NCCL process group of
    one rank (reduce-scatter over NCCL, device kernels), against the oracle."""
    import datetime
    import socket
    import torch
    import torch.distributed as tdist
    import spla_b200 as spla
    import spla_b200.distributed as sd
    from inputs import buffer
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    tdist.init_process_group("nccl", rank=0, world_size=1, init_method=f"tcp://127.0.0.1:{port}",
                             timeout=datetime.timedelta(seconds=60))
    try:
        dist = sd.Distribution.create_blacs_block_cyclic(None, "R", 1, 1, 16, 16)
        m, n, k = 50, 40, 20000
        dt = np.complex128
        A = buffer(dt, k, m, 1, "gauss_k", k)
        B = buffer(dt, k, n, 2, "gauss_k", k)
        C = buffer(dt, m + 3, n + 2, 3, "uniform11")
        dC = _dev(C)
        ctx = spla.Context(spla.PU_GPU)
        sd.pgemm_ssb(m, n, k, 2, 0.5 + 0.5j, _dev(A), k, _dev(B), k, -1.0, dC, m + 3, 2, 1, dist,
                     sd.DeviceBackend(ctx))
        torch.cuda.synchronize()
        ref = C.copy()
        assert oracle.pgemm_ssb(m, n, k, 2, 0.5 + 0.5j, A, k, B, k, -1.0, ref, m + 3, 2, 1) == 0
        assert oracle.rel_fro(dC.cpu().numpy(), ref) <= 1e-14
    finally:
        tdist.destroy_process_group()
