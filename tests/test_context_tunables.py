"""Context tunables against the reference library, on the CPU.

The reference's ContextInternal (src/spla/context_internal.hpp:58-64 defaults,
:122-140 setter validation) and its C ABI (src/spla/context.cpp:148-366) are
compared call by call with this library's: the default of every getter, the
return code of every setter for valid and invalid values (0, -1, the largest
int), the getters after each setter, null handles and null allocator
functions. Both contexts are host contexts (SPLA_PU_HOST), which neither
library creates on a device. The reference library is the one compiled from
its own sources (oracle/_ref); the test is skipped where it is absent.

Which tunables act in this library: tile_size_gpu bounds the k-chunk of
host-resident operands streamed to the device; num_tiles, tile_size_host and
op_threshold_gpu are kept and returned with the reference's validation but do
not change how a contraction runs (there is no host BLAS path and C is not
tiled over streams)."""
import ctypes as ct

import pytest

import oracle

INT_MAX = 2 ** 31 - 1
GETTERS = [("num_tiles", ct.c_int), ("tile_size_host", ct.c_int), ("tile_size_gpu", ct.c_int),
           ("op_threshold_gpu", ct.c_int), ("gpu_device_id", ct.c_int),
           ("allocated_memory_host", ct.c_uint64), ("allocated_memory_pinned", ct.c_uint64),
           ("allocated_memory_gpu", ct.c_uint64)]
SETTERS = ["num_tiles", "tile_size_host", "tile_size_gpu", "op_threshold_gpu"]
VALUES = [1, 7, 4096, 0, -1, INT_MAX, -INT_MAX - 1]


class Lib:
    def __init__(self, path):
        self.L = ct.CDLL(str(path))
        self.L.spla_ctx_create.argtypes = [ct.POINTER(ct.c_void_p), ct.c_int]
        self.L.spla_ctx_destroy.argtypes = [ct.POINTER(ct.c_void_p)]
        for name, _ in GETTERS:
            getattr(self.L, f"spla_ctx_{name}").argtypes = [ct.c_void_p, ct.c_void_p]
        for name in SETTERS:
            getattr(self.L, f"spla_ctx_set_{name}").argtypes = [ct.c_void_p, ct.c_int]
        for kind in ("host", "pinned", "gpu"):
            getattr(self.L, f"spla_ctx_set_alloc_{kind}").argtypes = [ct.c_void_p, ct.c_void_p,
                                                                     ct.c_void_p]

    def create(self):
        h = ct.c_void_p()
        assert self.L.spla_ctx_create(ct.byref(h), 0) == 0
        return h

    def destroy(self, h):
        return self.L.spla_ctx_destroy(ct.byref(h))

    def state(self, h):
        out = {}
        for name, ctype in GETTERS:
            v = ctype()
            rc = getattr(self.L, f"spla_ctx_{name}")(h, ct.byref(v))
            out[name] = (rc, v.value)
        return out

    def set(self, h, name, value):
        return getattr(self.L, f"spla_ctx_set_{name}")(h, value)


@pytest.fixture(scope="module")
def libs(spla_lib):
    if not oracle.REF_LIB.exists():
        pytest.skip("reference library not built (oracle/_ref)")
    return Lib(spla_lib.LIB_PATH), Lib(oracle.REF_LIB)


def test_defaults(libs):
    ours, ref = libs
    a, b = ours.create(), ref.create()
    try:
        sa, sb = ours.state(a), ref.state(b)
        assert sa == sb
        assert sa["num_tiles"] == (0, 4) and sa["tile_size_host"] == (0, 500)
        assert sa["tile_size_gpu"] == (0, 2048) and sa["op_threshold_gpu"] == (0, 2000000)
    finally:
        assert ours.destroy(a) == 0 and ref.destroy(b) == 0


@pytest.mark.parametrize("name", SETTERS)
def test_setters(libs, name):
    ours, ref = libs
    a, b = ours.create(), ref.create()
    try:
        for v in VALUES:
            ra, rb = ours.set(a, name, v), ref.set(b, name, v)
            assert ra == rb, (name, v, ra, rb)
            assert ours.state(a) == ref.state(b), (name, v)
    finally:
        ours.destroy(a)
        ref.destroy(b)


def test_null_handles(libs):
    ours, ref = libs
    for lib in (ours, ref):
        for name, ctype in GETTERS:
            v = ctype()
            assert getattr(lib.L, f"spla_ctx_{name}")(None, ct.byref(v)) == 5  # invalid handle
        for name in SETTERS:
            assert lib.set(None, name, 1) == 5


def test_null_allocator_functions(libs):
    """A null allocate or deallocate function is SPLA_INVALID_ALLOCATOR_FUNCTION
    (context.cpp:87-116) in both libraries."""
    ours, ref = libs
    libc = ct.CDLL(None)
    for lib in (ours, ref):
        h = lib.create()
        try:
            for kind in ("host", "pinned", "gpu"):
                f = getattr(lib.L, f"spla_ctx_set_alloc_{kind}")
                assert f(h, None, None) == 17
                assert f(h, ct.cast(libc.malloc, ct.c_void_p), None) == 17
                assert f(h, ct.cast(libc.malloc, ct.c_void_p), ct.cast(libc.free, ct.c_void_p)) == 0
        finally:
            lib.destroy(h)
