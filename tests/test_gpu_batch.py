"""Batched grouped contraction (splab_batch_*): uneven k, m, n in one
persistent launch replayed from a CUDA graph, against the oracle and against
one splab_gemm call per problem; autotuned and model-chosen k-chunks; graph
replays after the inputs change."""
import numpy as np
import pytest

import oracle
from inputs import buffer

pytestmark = pytest.mark.gpu


def _problems(torch, dt, shapes, seed):
    probs, host = [], []
    tdt = {np.complex128: torch.complex128, np.float64: torch.float64,
           np.complex64: torch.complex64, np.float32: torch.float32}[dt]
    for i, (m, n, k) in enumerate(shapes):
        A = buffer(dt, k, m, seed + 3 * i, "gauss_k", k)
        B = buffer(dt, k, n, seed + 3 * i + 1, "gauss_k", k)
        C = buffer(dt, m, n, seed + 3 * i + 2, "uniform11")
        dA, dB, dC = (torch.from_numpy(x).cuda() for x in (A, B, C))
        cplx = np.dtype(dt).kind == "c"
        alpha, beta = (1.0 - 0.5j, 0.25j) if cplx else (1.5, -0.5)
        probs.append(dict(opA=2 if cplx else 1, opB=0, m=m, n=n, k=k, A=dA, lda=k, B=dB, ldb=k,
                          C=dC, ldc=m, alpha=alpha, beta=beta))
        host.append((A, B, C, alpha, beta))
    return probs, host


@pytest.mark.parametrize("dt,tol,autotune", [(np.complex128, 1e-14, True),
                                             (np.float64, 1e-14, False),
                                             (np.complex64, 1e-6, True)])
def test_batch_matches_oracle(dt, tol, autotune):
    import torch
    import spla_b200 as spla
    shapes = [(130, 70, 9000), (64, 256, 4000), (200, 200, 12345), (17, 300, 2048),
              (256, 128, 30000), (96, 96, 777), (40, 40, 70000)]
    probs, host = _problems(torch, dt, shapes, 100)
    batch = spla.Batch(np.dtype(dt).name, probs)
    ws = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")
    batch.run(ws, autotune=autotune)
    torch.cuda.synchronize()
    info = batch.info()
    assert info["k_chunk"] in info["candidates"]
    if autotune:
        # every (tile, k-chunk) pair measured; the chosen pair is the fastest
        assert len(info["candidate_tiles"]) == len(info["tuning_ms"]) == len(info["candidates"])
        assert len(set(info["candidate_tiles"])) == 2
        assert all(t > 0 for t in info["tuning_ms"])
        best = int(np.argmin(info["tuning_ms"]))
        assert info["tile"] == info["candidate_tiles"][best]
        assert info["k_chunk"] == info["candidates"][best]
    else:
        assert info["tile"] in ((64, 64), (128, 64))
    for p, (A, B, C, alpha, beta) in zip(probs, host):
        ref = C.copy()
        assert oracle.pgemm_ssb(p["m"], p["n"], p["k"], p["opA"], alpha, A, p["k"], B, p["k"],
                                beta, ref, p["m"], 0, 0) == 0
        err = oracle.rel_fro(p["C"].cpu().numpy(), ref)
        assert err <= tol, (p["m"], p["n"], p["k"], err)


def test_batch_graph_replay_sees_new_inputs():
    """The captured graph reads the operands through their pointers: changing
    the input data between replays changes the result accordingly."""
    import torch
    import spla_b200 as spla
    shapes = [(128, 64, 5000), (96, 160, 7000)]
    probs, host = _problems(torch, np.complex128, shapes, 300)
    for p in probs:
        p["beta"] = 0.0
    batch = spla.Batch("complex128", probs)
    ws = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")
    batch.run(ws)
    first = [p["C"].clone() for p in probs]
    for p in probs:
        p["A"].mul_(2.0)
    batch.run(ws)
    batch.run(ws)
    torch.cuda.synchronize()
    for p, f in zip(probs, first):
        assert torch.allclose(p["C"], 2.0 * f, rtol=1e-13, atol=1e-16)


@pytest.mark.parametrize("dt,path,tol", [(np.complex64, 3, 1e-6), (np.float32, 3, 1e-6),
                                         (np.complex128, 2, 1e-14), (np.complex64, 2, 1e-6)])
def test_tensor_core_batch(dt, path, tol):
    """Batches on the 3xTF32 (path 3) and Ozaki (path 2) paths: the instances
    run in sequence with a shared workspace; the first run executes directly,
    the second captures the sequence in a CUDA graph and replays it, the third
    replays with changed inputs. Every result is checked against the oracle."""
    import torch
    import spla_b200 as spla
    shapes = [(130, 70, 9000), (300, 257, 20000), (17, 300, 2048), (256, 128, 30001)]
    probs, host = _problems(torch, dt, shapes, 500)
    for p in probs:
        p["beta"] = 0.0
    batch = spla.Batch(np.dtype(dt).name, probs, path=path)
    ws = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")

    def check(scale):
        torch.cuda.synchronize()
        batch.check(ws)
        for p, (A, B, C, alpha, beta) in zip(probs, host):
            ref = np.zeros_like(C)
            assert oracle.pgemm_ssb(p["m"], p["n"], p["k"], p["opA"], alpha * scale, A, p["k"],
                                    B, p["k"], 0.0, ref, p["m"], 0, 0) == 0
            err = oracle.rel_fro(p["C"].cpu().numpy(), ref)
            assert err <= tol, (p["m"], p["n"], p["k"], err)

    batch.run(ws)          # direct
    check(1.0)
    batch.run(ws)          # capture + replay
    check(1.0)
    for p in probs:
        p["A"].mul_(2.0)   # exact for floats
    batch.run(ws)          # replay sees the new data
    check(2.0)
    assert batch.info()["k_chunk"] == 0


def test_tensor_core_batch_rejects_unsupported():
    import torch
    import spla_b200 as spla
    probs, _ = _problems(torch, np.complex128, [(32, 32, 100)], 900)
    with pytest.raises(spla.InvalidParameterError):
        spla.Batch("complex128", probs, path=spla.PATH_TF32X3)  # 3xTF32 takes float dtypes


def test_batch_new_workspace_after_tuning():
    """A run with a different workspace than the tuning run uploads the work
    tables there before capturing: results stay correct."""
    import torch
    import spla_b200 as spla
    shapes = [(70, 90, 6000), (128, 32, 9000)]
    probs, host = _problems(torch, np.complex128, shapes, 700)
    for p in probs:
        p["beta"] = 0.0
    batch = spla.Batch("complex128", probs)
    ws1 = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")
    batch.run(ws1)
    ws2 = torch.full((batch.workspace_bytes,), 0xFF, dtype=torch.uint8, device="cuda")
    del ws1
    for p in probs:
        p["C"].zero_()
    batch.run(ws2)
    torch.cuda.synchronize()
    for p, (A, B, C, alpha, beta) in zip(probs, host):
        ref = np.zeros_like(C)
        assert oracle.pgemm_ssb(p["m"], p["n"], p["k"], p["opA"], alpha, A, p["k"], B, p["k"],
                                0.0, ref, p["m"], 0, 0) == 0
        assert oracle.rel_fro(p["C"].cpu().numpy(), ref) <= 1e-14


@pytest.mark.parametrize("opA,opB", [(0, 1), (2, 2)])
def test_ozaki_batch_in_place_operands(opA, opB):
    """Ozaki batches whose instances read op(A) = N or op(B) = T, C in place
    (m- and n-major rows through the transposing slicer): direct run, graph
    capture and replay, each instance checked against the device
    double-double product."""
    import torch
    import spla_b200 as spla
    g = torch.Generator(device="cuda")
    g.manual_seed(901)
    shapes = [(130, 70, 9000), (257, 300, 20000), (17, 300, 2048)]
    probs, refs = [], []
    for m, n, k in shapes:
        lda = m if opA == 0 else k
        ldb = k if opB == 0 else n
        s = (1.0 / (2 * k)) ** 0.5
        A = torch.randn(lda * (k if opA == 0 else m), dtype=torch.complex128, device="cuda",
                        generator=g) * s
        B = torch.randn(ldb * (n if opB == 0 else k), dtype=torch.complex128, device="cuda",
                        generator=g) * s
        C = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
        R = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
        assert spla.gemm_dd("complex128", opA, opB, m, n, k, A, lda, B, ldb, R, m) == 0
        probs.append(dict(opA=opA, opB=opB, m=m, n=n, k=k, A=A, lda=lda, B=B, ldb=ldb, C=C,
                          ldc=m, alpha=0.5 - 0.25j, beta=0.0))
        refs.append(R)
    batch = spla.Batch("complex128", probs, path=spla.PATH_OZAKI)
    ws = torch.empty(batch.workspace_bytes, dtype=torch.uint8, device="cuda")
    for _ in range(3):  # direct, capture + replay, replay
        for p in probs:
            p["C"].zero_()
        batch.run(ws)
        torch.cuda.synchronize()
        batch.check(ws)
        for p, R in zip(probs, refs):
            ref = (0.5 - 0.25j) * R
            err = float(torch.linalg.vector_norm(p["C"] - ref) / torch.linalg.vector_norm(ref))
            assert err <= 1e-14, (p["m"], p["n"], p["k"], err)
