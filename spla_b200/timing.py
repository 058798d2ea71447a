"""Per-phase timing of one local contraction through the kernel C ABI
(splab_gemm), device-resident operands, CUDA events on a private stream.

    python -m spla_b200.timing complex128:2:1024:1024:250000 [more specs]
    python -m spla_b200.timing --sweep     # every path and AUTO on a grid
    python -m spla_b200.timing --normalised complex128:2:1024:1024:250000

A spec is dtype:path:m:n:k[:opA[:opB]] with dtype in {float32, float64,
complex64, complex128} and path 0 auto, 1 DMMA, 2 Ozaki, 3 3xTF32; the
problem is C = op(A) op(B) with op(A) = conjugate transpose (complex) or
transpose (real) unless opA is given (0 = N: A is m x k, the pgemm_sbs
shape) and op(B) = N unless opB is given (1 = T, 2 = C: B is n x k), Gaussian
operands scaled by 1/sqrt(k), or with --normalised every row of op(A) and
column of B scaled to norm 1 (norms on a power of two: the rows whose
exponents the Ozaki path's one-pass scaling cannot estimate). One JSON line per spec: total time,
TFLOP/s and the phase times the path reports (scale/slice, GEMM span,
reduction or reconstruction, then one entry per GEMM launch) and, for the
Ozaki path, the parts of the slicing phase.
"""
from __future__ import annotations

import ctypes as ct
import json
import sys

NPHASE = 3 + 17


def run(dtype: str, path: int, m: int, n: int, k: int, steps: int = 5, warmup: int = 2,
        moduli: int = 0, opA: int | None = None, normalised: bool = False,
        opB: int = 0) -> dict:
    import torch
    import spla_b200 as spla
    L = spla.lib()
    tdt = getattr(torch, dtype)
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    A = torch.randn(m * k, dtype=tdt, device="cuda", generator=g) * (0.5 / k) ** 0.5
    B = torch.randn(n * k, dtype=tdt, device="cuda", generator=g) * (0.5 / k) ** 0.5
    C = torch.zeros(m * n, dtype=tdt, device="cuda")
    op = (2 if A.is_complex() else 1) if opA is None else opA
    if normalised:  # every row of op(A) and column of op(B) of norm 1
        Av = A.view(k, m).T if op == 0 else A.view(m, k)
        Av.div_(torch.linalg.vector_norm(Av, dim=1, keepdim=True))
        Bv = B.view(n, k) if opB == 0 else B.view(k, n).T
        Bv.div_(torch.linalg.vector_norm(Bv, dim=1, keepdim=True))
    lda = m if op == 0 else k
    ldb = k if opB == 0 else n
    ws_bytes = spla.splab_gemm_workspace_size(dtype, path, op, opB, m, n, k, moduli)
    ws = torch.empty(max(1, ws_bytes), dtype=torch.uint8, device="cuda")
    st = torch.cuda.Stream()
    pev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * NPHASE)]
    for e in pev:  # torch creates the CUDA event on first record
        e.record(st)
    st.synchronize()
    handles = (ct.c_void_p * (2 * NPHASE))(*[e.cuda_event for e in pev])

    def step():
        rc = spla.splab_gemm(dtype, path, op, opB, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, m,
                             moduli=moduli, workspace=ws, workspace_bytes=ws_bytes,
                             stream=st.cuda_stream)
        if rc != 0:
            raise RuntimeError(L.splab_status_string(rc).decode())

    with torch.cuda.stream(st):
        for _ in range(warmup):
            step()
        st.synchronize()
        tot = [0.0] * NPHASE
        ms = 0.0
        for _ in range(steps):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            for e in pev:
                e.record(st)  # phases a path does not have read as zero
            L.splab_set_phase_events(handles, NPHASE)
            try:
                t0.record(st)
                step()
                t1.record(st)
            finally:
                L.splab_set_phase_events(None, 0)
            st.synchronize()
            ms += t0.elapsed_time(t1)
            for p in range(NPHASE):
                tot[p] += pev[2 * p].elapsed_time(pev[2 * p + 1])
    ms /= steps
    ph = [x / steps for x in tot]
    flops = (8.0 if A.is_complex() else 2.0) * m * n * k
    return {"dtype": dtype, "path": path,
            "resolved_path": L.splab_gemm_path(spla._dtype_of(dtype=dtype), path, op, opB, m, n, k),
            "opA": op, "opB": opB, "m": m, "n": n, "k": k, "ms": round(ms, 3), "tflops": round(flops / ms / 1e9, 1),
            "phases_ms": [round(x, 3) for x in ph[:3]],
            "gemm_launch_ms": [round(x, 3) for x in ph[3:15] if x > 0.05],
            "slicing_ms": {"a_copy": round(ph[15], 3), "norms": round(ph[16], 3),
                           "residues_a": round(ph[17], 3), "residues_b": round(ph[18], 3),
                           "onepass_redo": round(ph[19], 3)},
            "workspace_GB": round(ws_bytes / 1e9, 2), "normalised": normalised}


def sweep():
    """Every path and AUTO's choice on a grid of square ssb problems: one JSON
    line per (dtype, m = n, k) with the time (ms) of each path."""
    for dt in ("complex128", "float64", "complex64", "float32"):
        paths = (0, 1, 2) if dt in ("complex128", "float64") else (0, 1, 2, 3)
        for (m, k) in [(128, 8192), (256, 8192), (256, 32768), (512, 16384), (512, 65536),
                       (1024, 16384), (2048, 8192)]:
            row = {"dtype": dt, "m": m, "n": m, "k": k}
            for p in paths:
                r = run(dt, p, m, m, k, steps=3, warmup=1)
                row[f"ms_path{p}"] = r["ms"]
                if p == 0:
                    row["auto_resolves_to"] = r["resolved_path"]
            print(json.dumps(row), flush=True)


def main(argv):
    if argv == ["--sweep"]:
        sweep()
        return
    normalised = "--normalised" in argv
    for spec in (a for a in argv if a != "--normalised"):
        d, p, m, n, k, *op = spec.split(":")
        print(json.dumps(run(d, int(p), int(m), int(n), int(k),
                             opA=int(op[0]) if op else None, normalised=normalised,
                             opB=int(op[1]) if len(op) > 1 else 0)), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["complex128:2:1024:1024:20000"])
