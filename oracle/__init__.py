"""ORACLE - test infrastructure only.

Python access to the CPU checkers built by oracle/Makefile:
  * liboracle.so  - the C restatement of the single-rank path with a
                    compensated (Dot2) accumulator (oracle.c);
  * _ref/libspla_ref.so - the unmodified reference host library, compiled from
                    its own sources when they are present (not on GPU boxes).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as ct
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libspla_ref.so"
DTYPE_CODE = {np.dtype(np.float32): 0, np.dtype(np.float64): 1, np.dtype(np.complex64): 2,
              np.dtype(np.complex128): 3}

_lib = None


def build(quiet: bool = True) -> None:
    """Compile the checkers (make in oracle/); _ref only where the reference exists."""
    out = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib() -> ct.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = ct.CDLL(str(LIB))
        L, vp, l_, i = _lib, ct.c_void_p, ct.c_long, ct.c_int
        L.oracle_gemm.argtypes = [i, i, i, l_, l_, l_, vp, vp, l_, vp, l_, vp, vp, l_, vp]
        L.oracle_gemm.restype = i
        L.oracle_pgemm_ssb.argtypes = [i, i, i, i, i, vp, vp, i, vp, i, vp, vp, i, i, i]
        L.oracle_pgemm_ssb.restype = i
        L.oracle_pgemm_sbs.argtypes = [i, i, i, i, vp, vp, i, vp, i, i, i, vp, vp, i, i]
        L.oracle_pgemm_sbs.restype = i
        L.oracle_block_info.argtypes = [l_] * 9 + [ct.POINTER(l_)]
        L.oracle_num_blocks.argtypes = [l_] * 6
        L.oracle_num_blocks.restype = l_
        L.oracle_block_is_active.argtypes = [l_] * 6 + [i]
        L.oracle_block_is_active.restype = i
        L.oracle_local_size.argtypes = [l_] * 4
        L.oracle_local_size.restype = l_
    return _lib


def _scalar(v, dt):
    dt = np.dtype(dt)
    if dt.kind == "c":
        return np.array([complex(v).real, complex(v).imag],
                        dtype=np.float32 if dt == np.complex64 else np.float64)
    return np.array([float(np.real(v))], dtype=np.float32 if dt == np.float32 else np.float64)


def _p(x):
    return None if x is None else x.ctypes.data


def _dt(*bufs):
    return next(x.dtype for x in bufs if x is not None)


def gemm(opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C_lo=None):
    """C <- alpha op(A) op(B) + beta C in double-double; C updated in place.
    A, B, C are flat column-major numpy buffers of one dtype. Returns the code."""
    dt = _dt(C, A, B)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    return lib().oracle_gemm(DTYPE_CODE[dt], opA, opB, m, n, k, _p(a), _p(A), lda, _p(B), ldb,
                             _p(b), _p(C), ldc, _p(C_lo))


def pgemm_ssb(m, n, k, opA, alpha, A, lda, B, ldb, beta, C, ldc, ro, co):
    dt = _dt(C, A, B)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    return lib().oracle_pgemm_ssb(DTYPE_CODE[dt], m, n, k, opA, _p(a), _p(A), lda, _p(B), ldb,
                                  _p(b), _p(C), ldc, ro, co)


def pgemm_sbs(mloc, n, k, alpha, A, lda, B, ldb, bro, bco, beta, C, ldc, gpu_order=1):
    dt = _dt(C, A, B)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    return lib().oracle_pgemm_sbs(DTYPE_CODE[dt], mloc, n, k, _p(a), _p(A), lda, _p(B), ldb, bro,
                                  bco, _p(b), _p(C), ldc, gpu_order)


def block_info(rb, cb, gr, gc, nr, nc, ro, co, idx):
    out = (ct.c_long * 9)()
    lib().oracle_block_info(rb, cb, gr, gc, nr, nc, ro, co, idx, out)
    return list(out)


def num_blocks(rb, cb, nr, nc, ro, co):
    return lib().oracle_num_blocks(rb, cb, nr, nc, ro, co)


def block_is_active(row, col, nrows, ncols, ro, co, mode):
    return bool(lib().oracle_block_is_active(row, col, nrows, ncols, ro, co, mode))


def local_size(global_size, block, proc, nprocs):
    return lib().oracle_local_size(global_size, block, proc, nprocs)


def rel_fro(x, ref):
    """Relative Frobenius error ||x - ref|| / ||ref|| (complex-aware), in float64."""
    x = np.asarray(x).astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    ref = np.asarray(ref).astype(x.dtype)
    den = np.linalg.norm(ref.ravel())
    num = np.linalg.norm((x - ref).ravel())
    return float(num / den) if den > 0 else float(num)
