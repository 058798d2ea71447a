"""Test helper: call any library that exports the spla_* C ABI through ctypes.

Used for the reference library compiled from its own sources
(oracle/_ref/libspla_ref.so, test infrastructure) and for this repository's
libspla.so with the same calls, so parity tests read the same on both sides.
Buffers are numpy arrays (host) or integer device addresses.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

MPI_COMM_SELF = 0x44000001
PREFIX = {np.float32: "s", np.float64: "d", np.complex64: "c", np.complex128: "z"}


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return x.data_ptr()  # torch tensor


class SplaCAPI:
    def __init__(self, path):
        self.lib = ct.CDLL(str(path))
        L, vp, i = self.lib, ct.c_void_p, ct.c_int
        L.spla_ctx_create.argtypes = [ct.POINTER(vp), i]
        L.spla_ctx_destroy.argtypes = [ct.POINTER(vp)]
        L.spla_mat_dis_create_block_cyclic.argtypes = [ct.POINTER(vp), i, ct.c_char, i, i, i, i]
        L.spla_mat_dis_create_mirror.argtypes = [ct.POINTER(vp), i]
        L.spla_mat_dis_destroy.argtypes = [ct.POINTER(vp)]
        for p, real in (("s", ct.c_float), ("d", ct.c_double), ("c", None), ("z", None)):
            sc = real if real is not None else vp
            getattr(L, f"spla_p{p}gemm_ssb").argtypes = [i, i, i, i, sc, vp, i, vp, i, sc, vp, i,
                                                        i, i, vp, vp]
            getattr(L, f"spla_p{p}gemm_ssbtr").argtypes = [i, i, i, i, sc, vp, i, vp, i, sc, vp,
                                                          i, i, i, i, vp, vp]
            getattr(L, f"spla_p{p}gemm_sbs").argtypes = [i, i, i, sc, vp, i, vp, i, i, i, vp, sc,
                                                        vp, i, vp]
            getattr(L, f"spla_{p}gemm").argtypes = [i, i, i, i, i, sc, vp, i, vp, i, sc, vp, i, vp]

    # handles -------------------------------------------------------------
    def ctx(self, pu):
        h = ct.c_void_p()
        rc = self.lib.spla_ctx_create(ct.byref(h), pu)
        assert rc == 0, rc
        return h

    def destroy_ctx(self, h):
        return self.lib.spla_ctx_destroy(ct.byref(h))

    def block_cyclic(self, rows=1, cols=1, rb=64, cb=64, order=b"R", comm=MPI_COMM_SELF):
        h = ct.c_void_p()
        rc = self.lib.spla_mat_dis_create_block_cyclic(ct.byref(h), comm, order, rows, cols, rb, cb)
        return rc, h

    def mirror(self, comm=MPI_COMM_SELF):
        h = ct.c_void_p()
        rc = self.lib.spla_mat_dis_create_mirror(ct.byref(h), comm)
        return rc, h

    # scalars -------------------------------------------------------------
    @staticmethod
    def _sc(v, dt):
        if dt in (np.float32,):
            return ct.c_float(float(np.real(v)))
        if dt in (np.float64,):
            return ct.c_double(float(np.real(v)))
        v = complex(v)
        ctype = ct.c_float if dt == np.complex64 else ct.c_double
        arr = (ctype * 2)(v.real, v.imag)
        return ct.cast(arr, ct.c_void_p), arr

    def _args(self, alpha, beta, dt):
        a, b = self._sc(alpha, dt), self._sc(beta, dt)
        keep = []
        if isinstance(a, tuple):
            keep += [a[1], b[1]]
            a, b = a[0], b[0]
        return a, b, keep

    # compute -------------------------------------------------------------
    def pgemm_ssb(self, dt, m, n, k, opA, alpha, A, lda, B, ldb, beta, C, ldc, ro, co, dist, ctx):
        a, b, _keep = self._args(alpha, beta, dt)
        f = getattr(self.lib, f"spla_p{PREFIX[dt]}gemm_ssb")
        return f(m, n, k, opA, a, _ptr(A), lda, _ptr(B), ldb, b, _ptr(C), ldc, ro, co, dist, ctx)

    def pgemm_ssbtr(self, dt, m, n, k, opA, alpha, A, lda, B, ldb, beta, C, ldc, ro, co, fill,
                    dist, ctx):
        a, b, _keep = self._args(alpha, beta, dt)
        f = getattr(self.lib, f"spla_p{PREFIX[dt]}gemm_ssbtr")
        return f(m, n, k, opA, a, _ptr(A), lda, _ptr(B), ldb, b, _ptr(C), ldc, ro, co, fill, dist,
                 ctx)

    def pgemm_sbs(self, dt, mloc, n, k, alpha, A, lda, B, ldb, bro, bco, dist, beta, C, ldc, ctx):
        a, b, _keep = self._args(alpha, beta, dt)
        f = getattr(self.lib, f"spla_p{PREFIX[dt]}gemm_sbs")
        return f(mloc, n, k, a, _ptr(A), lda, _ptr(B), ldb, bro, bco, dist, b, _ptr(C), ldc, ctx)

    def gemm(self, dt, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ctx):
        a, b, _keep = self._args(alpha, beta, dt)
        f = getattr(self.lib, f"spla_{PREFIX[dt]}gemm")
        return f(opA, opB, m, n, k, a, _ptr(A), lda, _ptr(B), ldb, b, _ptr(C), ldc, ctx)
