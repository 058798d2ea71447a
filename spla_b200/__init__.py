"""Python mirror of the SPLA interface on top of libspla.so (B200, sm_100a).

The functions and classes follow the reference's C++ interface
(include/spla/pgemm_ssb.hpp, pgemm_ssbtr.hpp, pgemm_sbs.hpp, gemm.hpp,
context.hpp, matrix_distribution.hpp): same names, same argument order and
meaning. Matrices are column-major buffers given as torch tensors (CUDA or
CPU), numpy arrays, or raw integer addresses; leading dimensions are in
elements, as in the C interface. Errors raise the exception class named like
the reference's C++ exception for the returned SplaError code.

The library must have been built (``python -m spla_b200.build``); importing
this module fails loudly otherwise - there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libspla.so"

# enums (include/spla/types.h)
DIST_BLACS_BLOCK_CYCLIC, DIST_MIRROR = 0, 1
PU_HOST, PU_GPU = 0, 1
OP_NONE, OP_TRANSPOSE, OP_CONJ_TRANSPOSE = 0, 1, 2
FILL_MODE_FULL, FILL_MODE_UPPER, FILL_MODE_LOWER = 0, 1, 2
# single-rank communicators (MPICH handle encoding, as the library's stand-in)
MPI_COMM_WORLD, MPI_COMM_SELF = 0x44000000, 0x44000001
# contraction paths (PATH_TF32X3: float and complex float only)
PATH_AUTO, PATH_DMMA, PATH_OZAKI, PATH_TF32X3 = 0, 1, 2, 3


class GenericError(RuntimeError):
    code = 1


def _mk(name, code, base=GenericError):
    return type(name, (base,), {"code": code})


InternalError = _mk("InternalError", 2)
InvalidParameterError = _mk("InvalidParameterError", 3)
InvalidPointerError = _mk("InvalidPointerError", 4)
InvalidHandleError = _mk("InvalidHandleError", 5)
MPIError = _mk("MPIError", 6)
MPIAllocError = _mk("MPIAllocError", 7, MPIError)
MPIThreadSupportError = _mk("MPIThreadSupportError", 8, MPIError)
GPUError = _mk("GPUError", 9)
GPUSupportError = _mk("GPUSupportError", 10, GPUError)
GPUAllocationError = _mk("GPUAllocationError", 11, GPUError)
GPULaunchError = _mk("GPULaunchError", 12, GPUError)
GPUNoDeviceError = _mk("GPUNoDeviceError", 13, GPUError)
GPUInvalidValueError = _mk("GPUInvalidValueError", 14, GPUError)
GPUInvalidDevicePointerError = _mk("GPUInvalidDevicePointerError", 15, GPUError)
GPUBlasError = _mk("GPUBlasError", 16, GPUError)
InvalidAllocatorFunctionError = _mk("InvalidAllocatorFunctionError", 17)
_BY_CODE = {c.code: c for c in [GenericError, InternalError, InvalidParameterError,
                                 InvalidPointerError, InvalidHandleError, MPIError, MPIAllocError,
                                 MPIThreadSupportError, GPUError, GPUSupportError,
                                 GPUAllocationError, GPULaunchError, GPUNoDeviceError,
                                 GPUInvalidValueError, GPUInvalidDevicePointerError, GPUBlasError,
                                 InvalidAllocatorFunctionError]}


def check(code: int):
    if code != 0:
        raise _BY_CODE.get(code, GenericError)(f"SPLA error code {code}")


_lib = None


def lib() -> ct.CDLL:
    """The loaded libspla.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} not found: build it with `python -m spla_b200.build`")
        _lib = ct.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L):
    vp, i, i64, sz = ct.c_void_p, ct.c_int, ct.c_int64, ct.c_size_t
    L.splab_gemm.argtypes = [i, i, i, i, i64, i64, i64, vp, vp, i64, vp, i64, vp, vp, i64, i, i64,
                             i64, i, vp, sz, vp]
    L.splab_gemm.restype = i
    L.splab_gemm_workspace_size.argtypes = [i, i, i, i, i64, i64, i64, i]
    L.splab_gemm_path.argtypes = [i, i, i, i, i64, i64, i64]
    L.splab_gemm_path.restype = i
    L.splab_gemm_check.argtypes = [i, i, i, i, i64, i64, i64, i, vp, vp]
    L.splab_gemm_check.restype = i
    L.splab_set_phase_events.argtypes = [vp, i]
    L.splab_set_phase_events.restype = i
    L.splab_gemm_workspace_size.restype = sz
    L.splab_status_string.argtypes = [i]
    L.splab_status_string.restype = ct.c_char_p
    L.splab_block_cyclic_info.argtypes = [i64] * 8 + [vp, i64, vp, vp]
    L.splab_block_cyclic_info.restype = i
    for name in ["spla_ctx_create"]:
        getattr(L, name).argtypes = [ct.POINTER(vp), i]
    L.spla_ctx_destroy.argtypes = [ct.POINTER(vp)]
    L.spla_b200_ctx_set_fp64_path.argtypes = [vp, i, i]
    for nm in ["spla_mat_dis_destroy"]:
        getattr(L, nm).argtypes = [ct.POINTER(vp)]
    L.spla_mat_dis_create_block_cyclic.argtypes = [ct.POINTER(vp), i, ct.c_char, i, i, i, i]
    L.spla_mat_dis_create_blacs_block_cyclic_from_mapping.argtypes = [ct.POINTER(vp), i, vp, i,
                                                                      i, i, i]
    L.spla_mat_dis_create_mirror.argtypes = [ct.POINTER(vp), i]
    # compute entry points
    for p, real in (("s", ct.c_float), ("d", ct.c_double), ("c", None), ("z", None)):
        sc = real if real is not None else vp
        getattr(L, f"spla_p{p}gemm_ssb").argtypes = [i, i, i, i, sc, vp, i, vp, i, sc, vp, i, i, i,
                                                    vp, vp]
        getattr(L, f"spla_p{p}gemm_ssbtr").argtypes = [i, i, i, i, sc, vp, i, vp, i, sc, vp, i, i,
                                                      i, i, vp, vp]
        getattr(L, f"spla_p{p}gemm_sbs").argtypes = [i, i, i, sc, vp, i, vp, i, i, i, vp, sc, vp,
                                                    i, vp]
        getattr(L, f"spla_{p}gemm").argtypes = [i, i, i, i, i, sc, vp, i, vp, i, sc, vp, i, vp]


# ---------------------------------------------------------------------------
# buffers

_DT_CODES = {"float32": 0, "float64": 1, "complex64": 2, "complex128": 3}
_PREFIX = {0: "s", 1: "d", 2: "c", 3: "z"}


def _addr(x):
    """(address, dtype code or None) of a torch tensor, numpy array, int or None."""
    if x is None:
        return None, None
    if isinstance(x, int):
        return x, None
    mod = type(x).__module__
    if mod.startswith("torch"):
        return x.data_ptr(), _DT_CODES.get(str(x.dtype).replace("torch.", ""))
    if mod.startswith("numpy"):
        return x.ctypes.data, _DT_CODES.get(str(x.dtype))
    raise TypeError(f"unsupported buffer type {type(x)}")


def _dtype_of(*bufs, dtype=None):
    if dtype is not None:
        return _DT_CODES[dtype] if isinstance(dtype, str) else int(dtype)
    for b in bufs:
        _, d = _addr(b)
        if d is not None:
            return d
    raise TypeError("cannot infer the dtype: pass dtype=")


def _scalar(v, dt):
    if dt == 0:
        return ct.c_float(float(v.real if isinstance(v, complex) else v))
    if dt == 1:
        return ct.c_double(float(v.real if isinstance(v, complex) else v))
    v = complex(v)
    arr = (ct.c_float * 2)(v.real, v.imag) if dt == 2 else (ct.c_double * 2)(v.real, v.imag)
    return arr


def _sarg(s, dt):
    return s if dt in (0, 1) else ct.cast(s, ct.c_void_p)


# ---------------------------------------------------------------------------
# Context / MatrixDistribution


class Context:
    """spla::Context (include/spla/context.hpp:58-196)."""

    def __init__(self, pu: int = PU_GPU):
        self._h = ct.c_void_p()
        check(lib().spla_ctx_create(ct.byref(self._h), int(pu)))

    @property
    def handle(self):
        return self._h

    def _get(self, name, ctype=ct.c_int):
        v = ctype()
        check(getattr(lib(), f"spla_ctx_{name}")(self._h, ct.byref(v)))
        return v.value

    def processing_unit(self):
        return self._get("processing_unit")

    def num_tiles(self):
        return self._get("num_tiles")

    def tile_size_host(self):
        return self._get("tile_size_host")

    def tile_size_gpu(self):
        return self._get("tile_size_gpu")

    def op_threshold_gpu(self):
        return self._get("op_threshold_gpu")

    def gpu_device_id(self):
        return self._get("gpu_device_id")

    def allocated_memory_host(self):
        return self._get("allocated_memory_host", ct.c_uint64)

    def allocated_memory_pinned(self):
        return self._get("allocated_memory_pinned", ct.c_uint64)

    def allocated_memory_gpu(self):
        return self._get("allocated_memory_gpu", ct.c_uint64)

    def set_num_tiles(self, v):
        check(lib().spla_ctx_set_num_tiles(self._h, int(v)))

    def set_tile_size_host(self, v):
        check(lib().spla_ctx_set_tile_size_host(self._h, int(v)))

    def set_tile_size_gpu(self, v):
        check(lib().spla_ctx_set_tile_size_gpu(self._h, int(v)))

    def set_op_threshold_gpu(self, v):
        check(lib().spla_ctx_set_op_threshold_gpu(self._h, int(v)))

    def set_fp64_path(self, path: int, moduli: int = 0):
        """Library extension: contraction path (PATH_AUTO / PATH_DMMA / PATH_OZAKI / PATH_TF32X3)."""
        check(lib().spla_b200_ctx_set_fp64_path(self._h, int(path), int(moduli)))

    def close(self):
        if self._h:
            check(lib().spla_ctx_destroy(ct.byref(self._h)))

    def __del__(self):
        try:
            if self._h:
                lib().spla_ctx_destroy(ct.byref(self._h))
        except Exception:
            pass


class MatrixDistribution:
    """spla::MatrixDistribution (include/spla/matrix_distribution.hpp:60-84)."""

    def __init__(self, handle):
        self._h = handle

    @staticmethod
    def create_blacs_block_cyclic(comm, order, proc_grid_rows, proc_grid_cols, row_block_size,
                                  col_block_size):
        h = ct.c_void_p()
        o = order.encode() if isinstance(order, str) else bytes([order])
        check(lib().spla_mat_dis_create_block_cyclic(ct.byref(h), int(comm), o,
                                                     int(proc_grid_rows), int(proc_grid_cols),
                                                     int(row_block_size), int(col_block_size)))
        return MatrixDistribution(h)

    @staticmethod
    def create_blacs_block_cyclic_from_mapping(comm, mapping, proc_grid_rows, proc_grid_cols,
                                               row_block_size, col_block_size):
        h = ct.c_void_p()
        arr = (ct.c_int * len(mapping))(*mapping) if mapping is not None else None
        check(lib().spla_mat_dis_create_blacs_block_cyclic_from_mapping(
            ct.byref(h), int(comm), arr, int(proc_grid_rows), int(proc_grid_cols),
            int(row_block_size), int(col_block_size)))
        return MatrixDistribution(h)

    @staticmethod
    def create_mirror(comm):
        h = ct.c_void_p()
        check(lib().spla_mat_dis_create_mirror(ct.byref(h), int(comm)))
        return MatrixDistribution(h)

    @property
    def handle(self):
        return self._h

    def _get(self, name):
        v = ct.c_int()
        check(getattr(lib(), f"spla_mat_dis_{name}")(self._h, ct.byref(v)))
        return v.value

    def proc_grid_rows(self):
        return self._get("proc_grid_rows")

    def proc_grid_cols(self):
        return self._get("proc_grid_cols")

    def row_block_size(self):
        return self._get("row_block_size")

    def col_block_size(self):
        return self._get("col_block_size")

    def type(self):
        return self._get("type")

    def comm(self):
        return self._get("comm")

    def set_row_block_size(self, v):
        check(lib().spla_mat_dis_set_row_block_size(self._h, int(v)))

    def set_col_block_size(self, v):
        check(lib().spla_mat_dis_set_col_block_size(self._h, int(v)))

    def __del__(self):
        try:
            if self._h:
                lib().spla_mat_dis_destroy(ct.byref(self._h))
        except Exception:
            pass


# ---------------------------------------------------------------------------
# compute entry points (argument order of the reference's C++ overloads)


def pgemm_ssb(m, n, kLocal, opA, alpha, A, lda, B, ldb, beta, C, ldc, cRowOffset, cColOffset,
              distC, ctx, dtype=None):
    """C <- alpha op(A) B + beta C, stripe x stripe -> block (pgemm_ssb.hpp:88-117)."""
    dt = _dtype_of(C, A, B, dtype=dtype)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    check(getattr(lib(), f"spla_p{_PREFIX[dt]}gemm_ssb")(
        m, n, kLocal, opA, _sarg(a, dt), _addr(A)[0], lda, _addr(B)[0], ldb, _sarg(b, dt),
        _addr(C)[0], ldc, cRowOffset, cColOffset, distC.handle, ctx.handle))


def pgemm_ssbtr(m, n, kLocal, opA, alpha, A, lda, B, ldb, beta, C, ldc, cRowOffset, cColOffset,
                cFillMode, distC, ctx, dtype=None):
    """pgemm_ssb limited to a triangle of C (pgemm_ssbtr.hpp:94-126)."""
    dt = _dtype_of(C, A, B, dtype=dtype)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    check(getattr(lib(), f"spla_p{_PREFIX[dt]}gemm_ssbtr")(
        m, n, kLocal, opA, _sarg(a, dt), _addr(A)[0], lda, _addr(B)[0], ldb, _sarg(b, dt),
        _addr(C)[0], ldc, cRowOffset, cColOffset, cFillMode, distC.handle, ctx.handle))


def pgemm_sbs(mLocal, n, k, alpha, A, lda, B, ldb, bRowOffset, bColOffset, descB, beta, C, ldc,
              ctx, dtype=None):
    """C <- alpha A B + beta C, stripe x block -> stripe (pgemm_sbs.hpp:86-116)."""
    dt = _dtype_of(C, A, B, dtype=dtype)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    check(getattr(lib(), f"spla_p{_PREFIX[dt]}gemm_sbs")(
        mLocal, n, k, _sarg(a, dt), _addr(A)[0], lda, _addr(B)[0], ldb, bRowOffset, bColOffset,
        descB.handle, _sarg(b, dt), _addr(C)[0], ldc, ctx.handle))


def gemm(opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ctx, dtype=None):
    """Local C <- alpha op(A) op(B) + beta C (gemm.hpp:66-97)."""
    dt = _dtype_of(C, A, B, dtype=dtype)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    check(getattr(lib(), f"spla_{_PREFIX[dt]}gemm")(
        opA, opB, m, n, k, _sarg(a, dt), _addr(A)[0], lda, _addr(B)[0], ldb, _sarg(b, dt),
        _addr(C)[0], ldc, ctx.handle))


# ---------------------------------------------------------------------------
# kernel-level entry (splab C ABI), device buffers only


def splab_gemm(dtype, path, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, fill=0, ro=0,
               co=0, moduli=0, workspace=None, workspace_bytes=0, stream=0):
    """Direct call of splab_gemm (include/splab.h); returns the status code."""
    dt = _dtype_of(dtype=dtype)
    a, b = _scalar(alpha, dt), _scalar(beta, dt)
    return lib().splab_gemm(dt, path, opA, opB, m, n, k, ct.cast(ct.pointer(a), ct.c_void_p)
                            if dt in (0, 1) else ct.cast(a, ct.c_void_p), _addr(A)[0], lda,
                            _addr(B)[0], ldb, ct.cast(ct.pointer(b), ct.c_void_p)
                            if dt in (0, 1) else ct.cast(b, ct.c_void_p), _addr(C)[0], ldc, fill,
                            ro, co, moduli, _addr(workspace)[0], workspace_bytes, stream)


def gemm_dd(dtype, opA, opB, m, n, k, A, lda, B, ldb, R_hi, ldr, R_lo=None, stream=0):
    """Double-double reference product R = op(A) op(B) on the device
    (splab_gemm_dd; verification only). R_hi / R_lo: device float64 (real) or
    complex128 (complex) buffers. Returns the status code."""
    L = lib()
    L.splab_gemm_dd.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_int64, ct.c_int64, ct.c_int64,
                                ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_int64, ct.c_void_p,
                                ct.c_void_p, ct.c_int64, ct.c_void_p]
    L.splab_gemm_dd.restype = ct.c_int
    return L.splab_gemm_dd(_dtype_of(dtype=dtype), opA, opB, m, n, k, _addr(A)[0], lda,
                           _addr(B)[0], ldb, _addr(R_hi)[0], _addr(R_lo)[0], ldr, stream)


def splab_gemm_workspace_size(dtype, path, opA, opB, m, n, k, moduli=0):
    return lib().splab_gemm_workspace_size(_dtype_of(dtype=dtype), path, opA, opB, m, n, k,
                                           moduli)


def splab_gemm_check(dtype, path, opA, opB, m, n, k, moduli=0, workspace=None, stream=0):
    return lib().splab_gemm_check(_dtype_of(dtype=dtype), path, opA, opB, m, n, k, moduli,
                                  _addr(workspace)[0], stream)


# ---------------------------------------------------------------------------
# batched grouped contraction (splab_batch_*)


class _Problem(ct.Structure):
    _fields_ = [("opA", ct.c_int), ("opB", ct.c_int), ("m", ct.c_int64), ("n", ct.c_int64),
                ("k", ct.c_int64), ("A", ct.c_void_p), ("lda", ct.c_int64), ("B", ct.c_void_p),
                ("ldb", ct.c_int64), ("C", ct.c_void_p), ("ldc", ct.c_int64),
                ("alpha", ct.c_double * 2), ("beta", ct.c_double * 2)]


class Batch:
    """A batch of independent local GEMMs of one dtype and op pair
    (splab_batch_*). path PATH_DMMA (default): one persistent grouped launch
    replayed from a CUDA graph; PATH_OZAKI / PATH_TF32X3: the instances in
    sequence on one stream with a shared workspace, replayed from a CUDA graph
    after the first run.

    problems: list of dicts with keys opA, opB, m, n, k, A, lda, B, ldb, C, ldc,
    alpha, beta (buffers as device tensors or integer addresses)."""

    def __init__(self, dtype, problems, path=None):
        L = lib()
        L.splab_batch_create_path.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p,
                                              ct.POINTER(ct.c_void_p), ct.POINTER(ct.c_size_t)]
        L.splab_batch_check.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p]
        L.splab_batch_run.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_size_t, ct.c_int,
                                      ct.c_void_p]
        L.splab_batch_info.argtypes = [ct.c_void_p, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int),
                                       ct.c_void_p, ct.c_void_p]
        L.splab_batch_destroy.argtypes = [ct.c_void_p]
        self.dtype = _dtype_of(dtype=dtype)
        arr = (_Problem * len(problems))()
        for i, p in enumerate(problems):
            a, b = complex(p.get("alpha", 1.0)), complex(p.get("beta", 0.0))
            arr[i] = _Problem(p["opA"], p["opB"], p["m"], p["n"], p["k"], _addr(p["A"])[0],
                              p["lda"], _addr(p["B"])[0], p["ldb"], _addr(p["C"])[0], p["ldc"],
                              (ct.c_double * 2)(a.real, a.imag), (ct.c_double * 2)(b.real, b.imag))
        self._arr = arr
        self._plan = ct.c_void_p()
        ws = ct.c_size_t()
        self.path = PATH_DMMA if path is None else int(path)
        rc = L.splab_batch_create_path(self.dtype, self.path, len(problems),
                                       ct.cast(arr, ct.c_void_p), ct.byref(self._plan),
                                       ct.byref(ws))
        if rc != 0:
            raise InvalidParameterError(
                f"splab_batch_create_path: {L.splab_status_string(rc).decode()}")
        self.workspace_bytes = ws.value

    def run(self, workspace, stream=0, autotune=True):
        rc = lib().splab_batch_run(self._plan, _addr(workspace)[0], self.workspace_bytes,
                                   int(bool(autotune)), stream)
        if rc != 0:
            raise GPULaunchError(f"splab_batch_run: {lib().splab_status_string(rc).decode()}")

    def check(self, workspace, stream=0):
        """Synchronise and raise GPULaunchError if a bounded device wait gave up."""
        rc = lib().splab_batch_check(self._plan, _addr(workspace)[0], stream)
        if rc != 0:
            raise GPULaunchError(f"splab_batch_check: {lib().splab_status_string(rc).decode()}")

    def info(self):
        """Chosen k-chunk and CTA tile; per tuning entry its k-chunk, tile and
        measured time (ms)."""
        L = lib()
        kc, nc = ct.c_int64(), ct.c_int()
        cands = (ct.c_int64 * 32)()
        ms = (ct.c_double * 32)()
        L.splab_batch_info(self._plan, ct.byref(kc), ct.byref(nc), ct.cast(cands, ct.c_void_p),
                           ct.cast(ms, ct.c_void_p))
        L.splab_batch_tiles.argtypes = [ct.c_void_p] + [ct.c_void_p] * 5
        tm, tn, ne = ct.c_int(), ct.c_int(), ct.c_int()
        etm, etn = (ct.c_int * 32)(), (ct.c_int * 32)()
        L.splab_batch_tiles(self._plan, ct.byref(tm), ct.byref(tn), ct.byref(ne),
                            ct.cast(etm, ct.c_void_p), ct.cast(etn, ct.c_void_p))
        return {"k_chunk": kc.value, "tile": (tm.value, tn.value),
                "candidates": list(cands[:nc.value]), "tuning_ms": list(ms[:nc.value]),
                "candidate_tiles": list(zip(etm[:ne.value], etn[:ne.value]))}

    def __del__(self):
        try:
            if self._plan:
                lib().splab_batch_destroy(self._plan)
        except Exception:
            pass
