"""Device scratch through the caller's allocator (spla_ctx_set_alloc_gpu): a
failing allocator makes the call return SPLA_GPU_ALLOCATION_ERROR (no crash,
C untouched, the context stays usable); a working allocator supplied by the
caller is used for the scratch, gives the oracle's result, and gets every
buffer back when the context is destroyed. Allocation failure is injected on
the host; nothing faults on the GPU."""
import ctypes as ct

import numpy as np
import pytest

import oracle
import spla_b200 as spla
from inputs import buffer

pytestmark = pytest.mark.gpu

ALLOC = ct.CFUNCTYPE(ct.c_void_p, ct.c_size_t)
FREE = ct.CFUNCTYPE(None, ct.c_void_p)


def test_caller_allocator_failure_and_success():
    import torch
    L = spla.lib()
    L.spla_ctx_set_alloc_gpu.argtypes = [ct.c_void_p, ALLOC, FREE]
    m, n, k = 64, 48, 120000  # long k: the FP64 path splits k and needs scratch
    A = buffer(np.complex128, k, m, 1, "gauss_k", k)
    B = buffer(np.complex128, k, n, 2, "gauss_k", k)
    C = buffer(np.complex128, m, n, 3, "uniform11")
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    d = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R", 1, 1, 64, 64)

    live = {}
    calls = {"alloc": 0, "free": 0, "fail": True}

    def alloc(size):
        calls["alloc"] += 1
        if calls["fail"]:
            return None
        p = torch.cuda.caching_allocator_alloc(int(size))
        live[p] = size
        return p

    def free(p):
        calls["free"] += 1
        torch.cuda.caching_allocator_delete(p)
        live.pop(p)

    alloc_cb, free_cb = ALLOC(alloc), FREE(free)  # kept alive for the context's lifetime
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_DMMA)
    assert L.spla_ctx_set_alloc_gpu(ctx.handle, alloc_cb, free_cb) == 0

    dC = torch.from_numpy(C).cuda()
    with pytest.raises(spla.GPUAllocationError):
        spla.pgemm_ssb(m, n, k, 2, 1.0, dA, k, dB, k, 0.0, dC, m, 0, 0, d, ctx)
    assert calls["alloc"] >= 1
    assert np.array_equal(dC.cpu().numpy(), C)  # C untouched

    calls["fail"] = False
    spla.pgemm_ssb(m, n, k, 2, 1.0, dA, k, dB, k, 0.0, dC, m, 0, 0, d, ctx)
    torch.cuda.synchronize()
    assert live, "the scratch came from the caller's allocator"
    ref = C.copy()
    assert oracle.pgemm_ssb(m, n, k, 2, 1.0, A, k, B, k, 0.0, ref, m, 0, 0) == 0
    assert oracle.rel_fro(dC.cpu().numpy(), ref) <= 1e-14

    del ctx
    import gc
    gc.collect()
    assert not live and calls["free"] >= 1
