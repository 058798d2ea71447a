"""Thin torch binding of the stripe-stripe-block contraction with a
hand-written adjoint.

    C = A^H B   (complex)  /  A^T B   (real)

with A (k x m) and B (k x n) stored column-major with k contiguous - the
layout of pgemm_ssb - which as torch tensors are row-major (m, k) and (n, k).
Forward: spla_p?gemm_ssb on the GPU. Backward (torch's convention for complex
gradients, grad = dL/d conj(z) * 2):

    dA = B . dC^H      (k x m)
    dB = A . dC        (k x n)

both computed with the stripe-block-stripe kernels (spla_p?gemm_sbs), which
take no op flag on B, so dC^H is formed explicitly (it is only m x n).
"""
from __future__ import annotations

import torch

import spla_b200 as spla

_DIST = {}


def _dist():
    key = torch.cuda.current_device()
    if key not in _DIST:
        _DIST[key] = spla.MatrixDistribution.create_blacs_block_cyclic(spla.MPI_COMM_SELF, "R",
                                                                       1, 1, 128, 128)
    return _DIST[key]


def ssb(A: torch.Tensor, B: torch.Tensor, ctx: "spla.Context") -> torch.Tensor:
    """C (m x n, returned as a column-major buffer viewed (n, m).T) = op(A) B with
    A given as (m, k) and B as (n, k) contiguous CUDA tensors."""
    m, k = A.shape
    n = B.shape[0]
    C = torch.empty((n, m), dtype=A.dtype, device=A.device)  # column-major m x n
    op = spla.OP_CONJ_TRANSPOSE if A.is_complex() else spla.OP_TRANSPOSE
    spla.pgemm_ssb(m, n, k, op, 1.0, A, k, B, k, 0.0, C, m, 0, 0, _dist(), ctx)
    return C.T


def sbs(A_cm: torch.Tensor, mloc: int, kk: int, B_cm: torch.Tensor, n: int, ctx) -> torch.Tensor:
    """C (mloc x n) = A (mloc x kk) . B (kk x n); all column-major buffers
    given as row-major tensors of shape (cols, rows)."""
    C = torch.empty((n, mloc), dtype=A_cm.dtype, device=A_cm.device)
    spla.pgemm_sbs(mloc, n, kk, 1.0, A_cm, mloc, B_cm, kk, 0, 0, _dist(), 0.0, C, mloc, ctx)
    return C


class SsbFunction(torch.autograd.Function):
    """C = A^H B with the adjoint on the sbs kernels (see module docstring)."""

    @staticmethod
    def forward(ctx_, A, B, spla_ctx):
        ctx_.save_for_backward(A, B)
        ctx_.spla_ctx = spla_ctx
        return ssb(A.contiguous(), B.contiguous(), spla_ctx)

    @staticmethod
    def backward(ctx_, dC):
        A, B = ctx_.saved_tensors
        sctx = ctx_.spla_ctx
        m, k = A.shape
        n = B.shape[0]
        dA = dB = None
        if ctx_.needs_input_grad[0]:
            # dA (k x m) = B (k x n) . dC^H (n x m); column-major buffers:
            # B is (n, k) row-major = k x n column-major; dC^H column-major n x m = (m, n) rows
            dCH = dC.conj().contiguous() if A.is_complex() else dC.contiguous()  # (m, n) = dC^H cm
            dA = sbs(B.contiguous(), k, n, dCH, m, sctx)  # (m, k) row-major = k x m cm
        if ctx_.needs_input_grad[1]:
            # dB (k x n) = A (k x m) . dC (m x n); dC column-major = dC.T rows (n, m)
            dCcm = dC.T.contiguous()
            dB = sbs(A.contiguous(), k, m, dCcm, n, sctx)  # (n, k) row-major = k x n cm
        return dA, dB, None


def ssb_autograd(A, B, spla_ctx):
    return SsbFunction.apply(A, B, spla_ctx)
