"""Multi-rank pgemm_ssb / pgemm_sbs: the reference's distributed operations,
one process per GPU, over a torch.distributed process group.

The reference distributes the long dimension k over MPI ranks ("stripes")
and moves blocks of C (ssb) or B (sbs) through ring engines
(src/pgemm_ssb/pgemm_ssb_gpu.cpp:75-240, src/pgemm_ssb/ring_ssb_gpu.cpp:118-516,
src/pgemm_sbs/pgemm_sbs_gpu.cpp:73-232, src/pgemm_sbs/ring_sbs_gpu.cpp:114-351).
Here every GPU sees every peer at full bandwidth through NVSwitch, so each
operation is one collective:

  pgemm_ssb:  every rank computes its partial C = op(A_r) B_r (m x n) with the
              local contraction (DMMA or Ozaki, as the context selects), packs
              it owner by owner in the block-cyclic map of C, and one
              reduce-scatter leaves on each owner the sum of its blocks, which
              it adds into its local C as alpha * sum + beta * C. A mirror C
              is one all-reduce and the same update on every rank.
  pgemm_sbs:  every rank packs the blocks of the k x n submatrix of B that it
              owns, one all-gather gives every rank all blocks, which it lays
              out as a dense k x n B, and the local contraction computes
              C = alpha A B + beta C on its rows. A mirror B needs no exchange.

The block map is the reference's BlockCyclicGenerator
(src/block_generation/block_cyclic_generator.cpp:59-141), evaluated by the
library's host code (splab_block_cyclic_blocks); the owner of grid index i is
the process rank mapping[i] of the distribution, with the ranks outside the
grid taking the remaining labels in order
(src/spla/matrix_distribution_internal.cpp:87-150). Block moves run on the
device (splab_copy_blocks). Collectives on complex data run on its real view.
Uneven owner segments are padded to the largest, so that the collectives
take equal chunks (NCCL reduce-scatter and all-gather).

Validation follows the reference: pgemm_ssb returns for m = 0 or n = 0, then
rejects op(A) = N and negative sizes or offsets, then checks the local sizes
(pgemm_ssb_host.cpp:151-171, :60-61); pgemm_sbs returns for k = 0 or n = 0,
runs locally for one rank or a mirror B, then rejects negative sizes or
offsets and checks the local sizes (pgemm_sbs_host.cpp:171-193, :77-79).

The device work goes through a `backend` object (`DeviceBackend`, the
library's kernels); the CPU tests pass a host backend so that the plans and
the collectives can be checked with gloo ranks without a GPU.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import (FILL_MODE_FULL, FILL_MODE_LOWER, FILL_MODE_UPPER, OP_NONE, OP_TRANSPOSE,
               OP_CONJ_TRANSPOSE, DIST_BLACS_BLOCK_CYCLIC, DIST_MIRROR, InvalidParameterError,
               InvalidPointerError, GPULaunchError, lib)

_CODE = {"float32": 0, "float64": 1, "complex64": 2, "complex128": 3}


# ---------------------------------------------------------------------------
# distributions over a process group


class Distribution:
    """A matrix distribution over a torch.distributed process group, with the
    factories and validation of spla::MatrixDistribution
    (include/spla/matrix_distribution.hpp:60-84,
    src/spla/matrix_distribution_internal.cpp:42-150)."""

    def __init__(self, kind, group, grid_rows, grid_cols, row_block, col_block, full_mapping):
        self.type = kind
        self.group = group
        self.proc_grid_rows = grid_rows
        self.proc_grid_cols = grid_cols
        self.row_block_size = row_block
        self.col_block_size = col_block
        # full_mapping[i]: process rank with grid index i (grid positions first,
        # then the ranks outside the grid)
        self.full_mapping = list(full_mapping)

    @staticmethod
    def _size_rank(group):
        import torch.distributed as dist
        return dist.get_world_size(group), dist.get_rank(group)

    @classmethod
    def create_blacs_block_cyclic(cls, group, order, rows, cols, rb, cb):
        if order not in ("R", "r", "C", "c"):
            raise InvalidParameterError("order must be R or C")
        if rows < 1 or cols < 1 or rb < 1 or cb < 1:
            raise InvalidParameterError("grid and block sizes must be >= 1")
        mapping = [0] * (rows * cols)
        counter = 0
        if order in ("R", "r"):
            for r in range(rows):
                for c in range(cols):
                    mapping[r + c * rows] = counter
                    counter += 1
        else:
            for c in range(cols):
                for r in range(rows):
                    mapping[r + c * rows] = counter
                    counter += 1
        return cls.create_blacs_block_cyclic_from_mapping(group, mapping, rows, cols, rb, cb)

    @classmethod
    def create_blacs_block_cyclic_from_mapping(cls, group, mapping, rows, cols, rb, cb):
        if rows < 1 or cols < 1 or rb < 1 or cb < 1:
            raise InvalidParameterError("grid and block sizes must be >= 1")
        if mapping is None:
            raise InvalidParameterError("mapping is null")
        size, _ = cls._size_rank(group)
        used = []
        for i in range(rows * cols):
            r = int(mapping[i])
            if r < 0 or r >= size or r in used:
                raise InvalidParameterError("mapping entries must be distinct ranks")
            used.append(r)
        full = used + [r for r in range(size) if r not in used]
        if len(full) != size:
            raise InvalidParameterError("grid larger than the process group")
        return cls(DIST_BLACS_BLOCK_CYCLIC, group, rows, cols, rb, cb, full)

    @classmethod
    def create_mirror(cls, group):
        size, _ = cls._size_rank(group)
        return cls(DIST_MIRROR, group, size, 1, 256, 256, list(range(size)))

    def comm_size(self):
        return len(self.full_mapping)

    def grid_index(self, rank=None):
        """The index of process `rank` (default: this process) in the grid order."""
        if rank is None:
            rank = self._size_rank(self.group)[1]
        return self.full_mapping.index(rank)

    def local_size(self, global_rows, global_cols, row_off, col_off, grid_idx):
        """Local rows and columns of grid index `grid_idx` for the submatrix
        (block_cyclic_generator.cpp:103-141)."""
        if self.type == DIST_MIRROR:
            return global_rows, global_cols
        R, C = self.proc_grid_rows, self.proc_grid_cols
        if grid_idx >= R * C:
            return 0, 0

        def ls(g, b, p, n):
            nb = g // b
            over = nb % n
            s = (nb // n) * b
            if p + 1 < over:
                s += b
            if p + 1 == over:
                s += g % b
            return s

        rows = (ls(global_rows + row_off, self.row_block_size, grid_idx % R, R) -
                ls(row_off, self.row_block_size, grid_idx % R, R))
        cols = (ls(global_cols + col_off, self.col_block_size, grid_idx // R, C) -
                ls(col_off, self.col_block_size, grid_idx // R, C))
        return rows, cols


# ---------------------------------------------------------------------------
# exchange plans


def block_map(dist, rows, cols, row_off, col_off):
    """(count, 9) int64 array of the block-cyclic map of the rows x cols
    submatrix at (row_off, col_off): global row, global col, sub-row, sub-col,
    local row, local col, rows, cols, owner grid index."""
    L = lib()
    L.splab_block_cyclic_blocks.argtypes = [ct.c_int64] * 8 + [ct.c_void_p]
    L.splab_block_cyclic_blocks.restype = ct.c_int64
    args = (dist.row_block_size, dist.col_block_size, dist.proc_grid_rows, dist.proc_grid_cols,
            rows, cols, row_off, col_off)
    n = L.splab_block_cyclic_blocks(*args, None)
    if n < 0:
        raise InvalidParameterError("bad block-cyclic map arguments")
    out = np.zeros((max(n, 0), 9), np.int64)
    if n:
        L.splab_block_cyclic_blocks(*args, out.ctypes.data)
    return out


def _active(sub_row, sub_col, nrows, ncols, row_off, col_off, fill):
    """block_is_active of the reference (src/block_generation/block.hpp:58-66)."""
    if fill == FILL_MODE_UPPER:
        return sub_col + ncols + col_off > sub_row + row_off
    if fill == FILL_MODE_LOWER:
        return sub_row + nrows + row_off > sub_col + col_off
    return True


class Plan:
    """Blocks grouped by owner process: `segments[p]` are the block rows of
    process p in pack order, `offsets` their element offsets inside the
    owner's segment, `seg` the padded segment length (elements)."""

    def __init__(self, blocks, owners, world):
        self.blocks = blocks
        self.world = world
        order = np.lexsort((np.arange(len(blocks)), owners)) if len(blocks) else np.zeros(0, int)
        self.segments = [[] for _ in range(world)]
        self.offsets = np.zeros(len(blocks), np.int64)
        fill = [0] * world
        for b in order:
            p = int(owners[b])
            self.segments[p].append(int(b))
            self.offsets[b] = fill[p]
            fill[p] += int(blocks[b, 6] * blocks[b, 7])
        self.used = fill
        self.seg = max(1, max(fill) if fill else 1)
        self.owner = owners
        self.max_block = int((blocks[:, 6] * blocks[:, 7]).max()) if len(blocks) else 0


def ssb_plan(dist, m, n, row_off, col_off, fill):
    blocks = block_map(dist, m, n, row_off, col_off)
    keep = np.array([_active(b[2], b[3], b[6], b[7], row_off, col_off, fill) for b in blocks],
                    bool) if len(blocks) else np.zeros(0, bool)
    blocks = blocks[keep]
    owners = np.array([dist.full_mapping[int(g)] for g in blocks[:, 8]], np.int64)
    return Plan(blocks, owners, dist.comm_size())


def sbs_plan(dist, k, n, row_off, col_off):
    blocks = block_map(dist, k, n, row_off, col_off)
    owners = np.array([dist.full_mapping[int(g)] for g in blocks[:, 8]], np.int64)
    return Plan(blocks, owners, dist.comm_size())


# Copy descriptors (srcOff, srcLd, dstOff, dstLd, rows, cols) of the exchange
# steps; a segment of the send buffer holds an owner's blocks one after the
# other, each column-major with its own row count as leading dimension.

def ssb_pack_desc(plan, m):
    """Dense m x n partial (ld m) -> the owner segments of the send buffer."""
    d = [[b[2] + b[3] * m, m, p * plan.seg + plan.offsets[i], b[6], b[6], b[7]]
         for p in range(plan.world) for i in plan.segments[p] for b in [plan.blocks[i]]]
    return np.array(d, np.int64).reshape(-1, 6)


def ssb_unpack_desc(plan, rank, ldc):
    """Process `rank`'s summed segment -> its local C (alpha, beta applied)."""
    d = [[plan.offsets[i], b[6], b[4] + b[5] * ldc, ldc, b[6], b[7]]
         for i in plan.segments[rank] for b in [plan.blocks[i]]]
    return np.array(d, np.int64).reshape(-1, 6)


def sbs_pack_desc(plan, rank, ldb):
    """Process `rank`'s local B -> its segment of the send buffer."""
    d = [[b[4] + b[5] * ldb, ldb, plan.offsets[i], b[6], b[6], b[7]]
         for i in plan.segments[rank] for b in [plan.blocks[i]]]
    return np.array(d, np.int64).reshape(-1, 6)


def sbs_unpack_desc(plan, k):
    """All gathered segments -> the dense k x n B (ld k)."""
    d = [[p * plan.seg + plan.offsets[i], b[6], b[2] + b[3] * k, k, b[6], b[7]]
         for p in range(plan.world) for i in plan.segments[p] for b in [plan.blocks[i]]]
    return np.array(d, np.int64).reshape(-1, 6)


# ---------------------------------------------------------------------------
# backends: where the partial products and the block moves run


class DeviceBackend:
    """The library's kernels on CUDA tensors: the local contraction through
    spla.gemm on the context's path, block moves through splab_copy_blocks."""

    def __init__(self, ctx):
        self.ctx = ctx

    def empty(self, like, count):
        import torch
        return torch.zeros(max(1, count), dtype=like.dtype, device=like.device)

    def product(self, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        from . import gemm
        gemm(opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, self.ctx,
             dtype=str(C.dtype).replace("torch.", ""))

    def copy_blocks(self, src, dst, desc, alpha, beta):
        import torch
        if len(desc) == 0:
            return
        # the kernel dereferences both buffers on the device: refuse host memory
        # here rather than hand a host address to the GPU
        for name, t in (("source", src), ("destination", dst)):
            if not (isinstance(t, torch.Tensor) and t.is_cuda):
                raise InvalidPointerError(f"block {name} must be a CUDA tensor")
        if src.dtype != dst.dtype:
            raise InvalidParameterError("block source and destination dtypes differ")
        dt = _CODE[str(dst.dtype).replace("torch.", "")]
        d = torch.from_numpy(np.ascontiguousarray(desc, np.int64)).to(dst.device)
        cplx = dt >= 2
        ctype = ct.c_float if dt in (0, 2) else ct.c_double
        a = (ctype * 2)(complex(alpha).real, complex(alpha).imag if cplx else 0.0)
        b = (ctype * 2)(complex(beta).real, complex(beta).imag if cplx else 0.0)
        L = lib()
        L.splab_copy_blocks.argtypes = [ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                        ct.c_int64, ct.c_int64, ct.c_void_p, ct.c_void_p,
                                        ct.c_void_p]
        L.splab_copy_blocks.restype = ct.c_int
        maxe = int((desc[:, 4] * desc[:, 5]).max())
        rc = L.splab_copy_blocks(dt, src.data_ptr(), dst.data_ptr(), d.data_ptr(), len(desc),
                                 maxe, ct.cast(a, ct.c_void_p), ct.cast(b, ct.c_void_p),
                                 torch.cuda.current_stream(dst.device).cuda_stream)
        if rc != 0:
            raise GPULaunchError(f"splab_copy_blocks: status {rc}")
        d.record_stream(torch.cuda.current_stream(dst.device))


# ---------------------------------------------------------------------------
# collectives (equal chunks; complex data on its real view)


def _real(t):
    import torch
    return torch.view_as_real(t) if t.is_complex() else t


def _reduce_scatter(send, recv, world, group):
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        dist.reduce_scatter_tensor(_real(recv), _real(send), group=group)
    else:  # gloo has no reduce-scatter: the same sums through an all-reduce
        dist.all_reduce(_real(send), group=group)
        me = dist.get_rank(group)
        recv.copy_(send[me * recv.numel():(me + 1) * recv.numel()])


def _all_gather(send, recv, group):
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        dist.all_gather_into_tensor(_real(recv), _real(send), group=group)
    else:
        world = dist.get_world_size(group)
        parts = list(_real(recv).chunk(world))
        dist.all_gather(parts, _real(send), group=group)


# ---------------------------------------------------------------------------
# operations


def _check_param(opA, opB, m, n, k, A, lda, B, ldb, C, ldc):
    """check_gemm_param (src/util/check_gemm_param.hpp:36-50)."""
    if m < 0 or n < 0 or k < 0:
        raise InvalidParameterError("negative size")
    if (opA == OP_NONE and lda < m) or (opA != OP_NONE and lda < k):
        raise InvalidParameterError("lda too small")
    if (opB == OP_NONE and ldb < k) or (opB != OP_NONE and ldb < n):
        raise InvalidParameterError("ldb too small")
    if k != 0 and m != 0 and A is None:
        raise InvalidPointerError("A is null")
    if k != 0 and n != 0 and B is None:
        raise InvalidPointerError("B is null")
    if n != 0 and m != 0 and C is None:
        raise InvalidPointerError("C is null")


def pgemm_ssb(m, n, kLocal, opA, alpha, A, lda, B, ldb, beta, C, ldc, cRowOffset, cColOffset,
              distC, backend, cFillMode=FILL_MODE_FULL):
    """C <- alpha op(A) B + beta C with A, B split along k over the ranks of
    distC's group (stripes of kLocal rows each) and C distributed by distC
    (block-cyclic: each rank passes its local C; mirror: the full C on every
    rank), the submatrix at (cRowOffset, cColOffset). Argument order of
    spla::pgemm_ssbtr (include/spla/pgemm_ssbtr.hpp:94-126); `backend` runs
    the local work (DeviceBackend(ctx) on GPUs)."""
    import torch.distributed as dist
    if m == 0 or n == 0:
        return
    if opA not in (OP_TRANSPOSE, OP_CONJ_TRANSPOSE):
        raise InvalidParameterError("op(A) must be transpose or conjugate transpose")
    if m < 0 or n < 0 or cRowOffset < 0 or cColOffset < 0:
        raise InvalidParameterError("negative size or offset")
    group = distC.group
    world = distC.comm_size()
    me = dist.get_rank(group)
    if distC.type == DIST_MIRROR:
        lr, lc = m, n
    else:
        lr, lc = distC.local_size(m, n, cRowOffset, cColOffset, distC.grid_index(me))
    _check_param(opA, OP_NONE, lr, lc, kLocal, A, lda, B, ldb, C, ldc)
    # the local partial product, m x n, dense (dtype and device of the first buffer given)
    like = next((x for x in (C, A, B) if x is not None), None)
    if like is None:
        raise InvalidPointerError("no buffer given")
    P = backend.empty(like, m * n)
    backend.product(opA, OP_NONE, m, n, kLocal, 1.0, A, lda, B, ldb, 0.0, P, m)
    if distC.type == DIST_MIRROR:
        dist.all_reduce(_real(P), group=group)
        if C is not None:
            desc = np.array([[0, m, cRowOffset + cColOffset * ldc, ldc, m, n]], np.int64)
            backend.copy_blocks(P, C, desc, alpha, beta)
        return
    plan = ssb_plan(distC, m, n, cRowOffset, cColOffset, cFillMode)
    send = backend.empty(P, world * plan.seg)
    backend.copy_blocks(P, send, ssb_pack_desc(plan, m), 1.0, 0.0)
    recv = backend.empty(P, plan.seg)
    _reduce_scatter(send, recv, world, group)
    if C is not None:
        backend.copy_blocks(recv, C, ssb_unpack_desc(plan, me, ldc), alpha, beta)


def pgemm_sbs(mLocal, n, k, alpha, A, lda, B, ldb, bRowOffset, bColOffset, descB, beta, C, ldc,
              backend):
    """C <- alpha A B + beta C with A, C split by rows over the ranks (stripes
    of mLocal rows) and B distributed by descB, the k x n submatrix at
    (bRowOffset, bColOffset). Argument order of spla::pgemm_sbs
    (include/spla/pgemm_sbs.hpp:86-116)."""
    import torch.distributed as dist
    if k == 0 or n == 0:
        return
    group = descB.group
    world = descB.comm_size()
    if world == 1 or descB.type == DIST_MIRROR:
        off = bRowOffset + bColOffset * ldb
        Bs = B[off:] if B is not None else None
        _check_param(OP_NONE, OP_NONE, mLocal, n, k, A, lda, Bs, ldb, C, ldc)
        backend.product(OP_NONE, OP_NONE, mLocal, n, k, alpha, A, lda, Bs, ldb, beta, C, ldc)
        return
    if n < 0 or k < 0 or bRowOffset < 0 or bColOffset < 0:
        raise InvalidParameterError("negative size or offset")
    me = dist.get_rank(group)
    lr, lc = descB.local_size(k, n, bRowOffset, bColOffset, descB.grid_index(me))
    _check_param(OP_NONE, OP_NONE, mLocal, lc, lr, A, lda, B, ldb, C, ldc)
    plan = sbs_plan(descB, k, n, bRowOffset, bColOffset)
    like = next((x for x in (C, A, B) if x is not None), None)
    if like is None:
        raise InvalidPointerError("no buffer given")
    send = backend.empty(like, plan.seg)
    if B is not None:
        backend.copy_blocks(B, send, sbs_pack_desc(plan, me, ldb), 1.0, 0.0)
    gathered = backend.empty(like, world * plan.seg)
    _all_gather(send, gathered, group)
    Bfull = backend.empty(like, k * n)
    backend.copy_blocks(gathered, Bfull, sbs_unpack_desc(plan, k), 1.0, 0.0)
    if mLocal > 0:
        backend.product(OP_NONE, OP_NONE, mLocal, n, k, alpha, A, lda, Bfull, k, beta, C, ldc)
