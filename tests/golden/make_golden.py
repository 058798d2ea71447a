"""Generate the golden fixtures in this folder from the REFERENCE library itself.

Runs the unmodified reference host library (compiled from its own sources into
oracle/_ref/libspla_ref.so by oracle/Makefile; needs the reference sources,
so it runs in the build container, not on GPU boxes) through its C ABI on
seeded inputs from tests/inputs.py and stores its outputs:

  gemm.npz / gemm.json      spla_?gemm grid of the reference's tests/test_gemm.cpp:240-254
                            (m,n,k in {1,13,32,263}, op in {N,C}, alpha=2, beta=3, padded lds)
  ssb.npz / ssb.json        spla_p?gemm_ssb / _ssbtr single-rank cases with C offsets
                            (tests/test_gemm_ssb.cpp:329-455 shapes), all four dtypes
  sbs.npz / sbs.json        spla_p?gemm_sbs single-rank cases with B offsets
  errors.json               SplaError codes of invalid calls
  index_map.npz             BlockCyclicGenerator block info / local sizes / fill predicate
  cfg1.npz                  pdgemm_ssb k=20000, m=n=256, op=T, U[-1,1] (full C)
  ref_symbols.txt           the spla_* C symbols the reference library exports

Outputs larger than 1024 elements are stored as a seeded sample of 128
entries of the C buffer (index, value). Usage:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

os.environ.setdefault("OPENBLAS_CORETYPE", "SkylakeX")

import oracle  # noqa: E402
from capi import SplaCAPI  # noqa: E402
from inputs import buffer, sample_indices  # noqa: E402

DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
FULL_LIMIT = 1024
SAMPLES = 128


def store(arrays, key, C, seed):
    if C.size <= FULL_LIMIT:
        arrays[key + "_idx"] = np.arange(C.size, dtype=np.int64)
        arrays[key + "_val"] = C.copy()
    else:
        idx = sample_indices(C.size, SAMPLES, seed).astype(np.int64)
        arrays[key + "_idx"] = idx
        arrays[key + "_val"] = C[idx].copy()


def gen_gemm(ref, ctx):
    cases, arrays = [], {}
    sizes = [1, 13, 32, 263]
    cid = 0
    for dtn in ("d", "z", "s", "c"):
        ops = [(0, 0), (0, 2), (2, 0), (2, 2)] if dtn in ("d", "z") else [(0, 0), (1, 0), (2, 2)]
        if dtn in ("z",):
            ops += [(1, 1), (1, 2), (2, 1)]
        sz = sizes if dtn in ("d", "z") else [1, 13, 263]
        for (opA, opB) in ops:
            for m in sz:
                for n in sz:
                    for k in sz:
                        dt = DT[dtn]
                        lda = (m if opA == 0 else k) + 5
                        ldb = (k if opB == 0 else n) + 6
                        ldc = m + 7
                        seed = 1000 + cid
                        A = buffer(dt, lda, k if opA == 0 else m, seed)
                        B = buffer(dt, ldb, n if opB == 0 else k, seed + 50000)
                        C = buffer(dt, ldc, n, seed + 90000)
                        rc = ref.gemm(dt, opA, opB, m, n, k, 2.0, A, lda, B, ldb, 3.0, C, ldc, ctx)
                        assert rc == 0, (dtn, opA, opB, m, n, k, rc)
                        store(arrays, f"c{cid}", C, seed)
                        cases.append(dict(id=cid, dtype=dtn, opA=opA, opB=opB, m=m, n=n, k=k,
                                          lda=lda, ldb=ldb, ldc=ldc, seed=seed, alpha=2.0,
                                          beta=3.0))
                        cid += 1
    return cases, arrays


def gen_ssb(ref, ctx):
    cases, arrays = [], {}
    cid = 0
    rc, dist = ref.block_cyclic(1, 1, 64, 64)
    assert rc == 0
    for dtn in ("d", "z", "s", "c"):
        dt = DT[dtn]
        cplx = dtn in ("c", "z")
        for (m, n) in [(1, 1), (13, 32), (32, 13), (263, 263), (100, 300)]:
            for k in (0, 1, 57, 400):
                for (ro, co) in [(0, 0), (2, 3)]:
                    for opA in ((1, 2) if cplx else (1,)):
                        for fill in (0, 1, 2):
                            if fill and (m, n) not in [(263, 263), (100, 300)]:
                                continue
                            lda, ldb = k + 3, k + 1
                            ldc = m + ro + 4
                            seed = 7000 + cid
                            A = buffer(dt, lda, m, seed)
                            B = buffer(dt, ldb, n, seed + 50000)
                            C = buffer(dt, ldc, n + co, seed + 90000)
                            alpha = (1.5 - 0.5j) if cplx else 1.5
                            beta = (0.5 + 0.25j) if cplx else 0.5
                            rc = ref.pgemm_ssbtr(dt, m, n, k, opA, alpha, A, lda, B, ldb, beta, C,
                                                 ldc, ro, co, fill, dist, ctx)
                            assert rc == 0, rc
                            store(arrays, f"c{cid}", C, seed)
                            cases.append(dict(id=cid, dtype=dtn, m=m, n=n, k=k, opA=opA, ro=ro,
                                              co=co, fill=fill, lda=lda, ldb=ldb, ldc=ldc,
                                              seed=seed, alpha=[np.real(alpha), np.imag(alpha)],
                                              beta=[np.real(beta), np.imag(beta)]))
                            cid += 1
    return cases, arrays


def gen_sbs(ref, ctx):
    cases, arrays = [], {}
    cid = 0
    rc, dist = ref.block_cyclic(1, 1, 128, 128)
    assert rc == 0
    for dtn in ("d", "z", "s", "c"):
        dt = DT[dtn]
        cplx = dtn in ("c", "z")
        for mloc in (1, 13, 263, 1000):
            for (n, k) in [(1, 1), (13, 32), (32, 13), (64, 200)]:
                for (bro, bco) in [(0, 0), (2, 3)]:
                    lda, ldc = mloc + 2, mloc + 5
                    ldb = k + bro + 3
                    seed = 9000 + cid
                    A = buffer(dt, lda, k, seed)
                    B = buffer(dt, ldb, n + bco, seed + 50000)
                    C = buffer(dt, ldc, n, seed + 90000)
                    alpha = (0.75 + 0.5j) if cplx else 0.75
                    beta = (1.0 - 0.5j) if cplx else 1.0
                    rc = ref.pgemm_sbs(dt, mloc, n, k, alpha, A, lda, B, ldb, bro, bco, dist,
                                       beta, C, ldc, ctx)
                    assert rc == 0, rc
                    store(arrays, f"c{cid}", C, seed)
                    cases.append(dict(id=cid, dtype=dtn, mloc=mloc, n=n, k=k, bro=bro, bco=bco,
                                      lda=lda, ldb=ldb, ldc=ldc, seed=seed,
                                      alpha=[np.real(alpha), np.imag(alpha)],
                                      beta=[np.real(beta), np.imag(beta)]))
                    cid += 1
    return cases, arrays


def gen_errors(ref, ctx):
    """Codes the reference returns for invalid calls (single rank, host context)."""
    rc, dist = ref.block_cyclic(1, 1, 64, 64)
    A = np.ones(1000, np.float64)
    B = np.ones(1000, np.float64)
    C = np.ones(1000, np.float64)
    d = np.float64
    out = []

    def rec(name, call, args):
        out.append(dict(name=name, call=call, args=args, code=int(rc_of(call, args))))

    def rc_of(call, a):
        if call == "ssb":
            return ref.pgemm_ssb(d, a["m"], a["n"], a["k"], a["opA"], 1.0,
                                 A if a.get("A", 1) else None, a["lda"],
                                 B if a.get("B", 1) else None, a["ldb"], 0.0,
                                 C if a.get("C", 1) else None, a["ldc"], a["ro"], a["co"], dist,
                                 ctx)
        if call == "sbs":
            return ref.pgemm_sbs(d, a["m"], a["n"], a["k"], 1.0, A if a.get("A", 1) else None,
                                 a["lda"], B if a.get("B", 1) else None, a["ldb"], a["bro"],
                                 a["bco"], dist, 0.0, C if a.get("C", 1) else None, a["ldc"], ctx)
        return ref.gemm(d, a["opA"], a["opB"], a["m"], a["n"], a["k"], 1.0,
                        A if a.get("A", 1) else None, a["lda"], B if a.get("B", 1) else None,
                        a["ldb"], 0.0, C if a.get("C", 1) else None, a["ldc"], ctx)

    base = dict(m=4, n=5, k=6, opA=1, lda=6, ldb=6, ldc=4, ro=0, co=0)
    rec("ssb ok", "ssb", base)
    rec("ssb opA none", "ssb", {**base, "opA": 0})
    rec("ssb m zero with bad op", "ssb", {**base, "m": 0, "opA": 0})
    rec("ssb n zero", "ssb", {**base, "n": 0})
    rec("ssb negative m", "ssb", {**base, "m": -1})
    rec("ssb negative k", "ssb", {**base, "k": -1})
    rec("ssb negative row offset", "ssb", {**base, "ro": -1})
    rec("ssb lda too small", "ssb", {**base, "lda": 5})
    rec("ssb ldb too small", "ssb", {**base, "ldb": 5})
    rec("ssb null A", "ssb", {**base, "A": 0})
    rec("ssb null B", "ssb", {**base, "B": 0})
    rec("ssb null C", "ssb", {**base, "C": 0})
    rec("ssb null A k zero", "ssb", {**base, "A": 0, "B": 0, "k": 0})
    sb = dict(m=4, n=5, k=6, lda=4, ldb=6, ldc=4, bro=0, bco=0)
    rec("sbs ok", "sbs", sb)
    rec("sbs k zero", "sbs", {**sb, "k": 0})
    rec("sbs lda too small", "sbs", {**sb, "lda": 3})
    rec("sbs ldb too small", "sbs", {**sb, "ldb": 5})
    rec("sbs negative m", "sbs", {**sb, "m": -2})
    rec("sbs null B", "sbs", {**sb, "B": 0})
    rec("sbs null C", "sbs", {**sb, "C": 0})
    g = dict(opA=0, opB=0, m=4, n=5, k=6, lda=4, ldb=6, ldc=4)
    rec("gemm ok", "gemm", g)
    rec("gemm ldc small is accepted", "gemm", {**g, "ldc": 1})
    rec("gemm lda too small NN", "gemm", {**g, "lda": 3})
    rec("gemm lda too small CN", "gemm", {**g, "opA": 2, "lda": 5})
    rec("gemm ldb too small NC", "gemm", {**g, "opB": 2, "ldb": 4})
    rec("gemm negative k", "gemm", {**g, "k": -1})
    rec("gemm null A", "gemm", {**g, "A": 0})
    rec("gemm m zero null all", "gemm", {**g, "m": 0, "A": 0, "B": 0, "C": 0})
    return out


def gen_index_map():
    """Block-cyclic mapping of the reference (src/block_generation/*) on random grids."""
    import ctypes as ct
    L = ct.CDLL(str(oracle.REF_LIB))
    l_ = ct.c_long
    L.ref_num_blocks.argtypes = [l_] * 8
    L.ref_num_blocks.restype = l_
    L.ref_block_info.argtypes = [l_] * 9 + [ct.POINTER(l_)]
    L.ref_local_rows.argtypes = [l_] * 9
    L.ref_local_rows.restype = l_
    L.ref_local_cols.argtypes = [l_] * 9
    L.ref_local_cols.restype = l_
    L.ref_block_is_active.argtypes = [l_] * 6 + [ct.c_int]
    L.ref_block_is_active.restype = ct.c_int
    rng = np.random.default_rng(424242)
    params, infos, local, active = [], [], [], []
    for _ in range(200):
        rb, cb = int(rng.integers(1, 70)), int(rng.integers(1, 70))
        gr, gc = int(rng.integers(1, 5)), int(rng.integers(1, 5))
        nr, nc = int(rng.integers(1, 400)), int(rng.integers(1, 400))
        ro, co = int(rng.integers(0, 150)), int(rng.integers(0, 150))
        nb = L.ref_num_blocks(rb, cb, gr, gc, nr, nc, ro, co)
        params.append([rb, cb, gr, gc, nr, nc, ro, co, nb])
        for b in range(min(nb, 64)):
            out = (l_ * 9)()
            L.ref_block_info(rb, cb, gr, gc, nr, nc, ro, co, b, out)
            infos.append([len(params) - 1, b] + list(out))
        for rank in range(gr * gc):
            local.append([len(params) - 1, rank, L.ref_local_rows(rb, cb, gr, gc, nr, nc, ro, co, rank),
                          L.ref_local_cols(rb, cb, gr, gc, nr, nc, ro, co, rank)])
    for _ in range(2000):
        row, col = int(rng.integers(0, 300)), int(rng.integers(0, 300))
        nrow, ncol = int(rng.integers(1, 80)), int(rng.integers(1, 80))
        ro, co = int(rng.integers(0, 50)), int(rng.integers(0, 50))
        mode = int(rng.integers(0, 3))
        active.append([row, col, nrow, ncol, ro, co, mode,
                       L.ref_block_is_active(row, col, nrow, ncol, ro, co, mode)])
    return dict(params=np.array(params, np.int64), infos=np.array(infos, np.int64),
                local=np.array(local, np.int64), active=np.array(active, np.int64))


def gen_cfg1(ref, ctx):
    """pdgemm_ssb k=20000, m=n=256, op=T, alpha=1, beta=0, U[-1,1] (full C)."""
    k, m, n = 20000, 256, 256
    A = buffer(np.float64, k, m, 20250001, "uniform11")
    B = buffer(np.float64, k, n, 20250001 + 1, "uniform11")
    C = np.zeros(m * n, np.float64)
    rc, dist = ref.block_cyclic(1, 1, 64, 64)
    assert ref.pgemm_ssb(np.float64, m, n, k, 1, 1.0, A, k, B, k, 0.0, C, m, 0, 0, dist, ctx) == 0
    return dict(C=C, k=np.int64(k), m=np.int64(m), n=np.int64(n))


def main():
    oracle.build()
    if not oracle.REF_LIB.exists():
        raise SystemExit("reference library not built (needs the reference sources)")
    ref = SplaCAPI(oracle.REF_LIB)
    ctx = ref.ctx(0)
    for name, fn in (("gemm", gen_gemm), ("ssb", gen_ssb), ("sbs", gen_sbs)):
        cases, arrays = fn(ref, ctx)
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        (HERE / f"{name}.json").write_text(json.dumps(cases, indent=0))
        print(name, len(cases), "cases")
    (HERE / "errors.json").write_text(json.dumps(gen_errors(ref, ctx), indent=1))
    np.savez_compressed(HERE / "index_map.npz", **gen_index_map())
    np.savez_compressed(HERE / "cfg1.npz", **gen_cfg1(ref, ctx))
    import subprocess
    nm = subprocess.run(["nm", "-D", "--defined-only", str(oracle.REF_LIB)], capture_output=True,
                        text=True, check=True).stdout
    syms = sorted({ln.split()[-1] for ln in nm.splitlines()
                   if " T " in ln and ln.split()[-1].startswith("spla_")})
    (HERE / "ref_symbols.txt").write_text("\n".join(syms) + "\n")
    ref.destroy_ctx(ctx)


if __name__ == "__main__":
    main()
