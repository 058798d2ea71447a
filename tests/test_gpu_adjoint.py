"""Differentiable ssb -> loss: C = A^H B (complex double, k = 100000,
m = n = 512, Gaussian / sqrt(k)), L = ||C - I||_F^2, with the hand-written
adjoint dA = B dC^H, dB = A dC on the sbs kernels behind
torch.autograd.Function (spla_b200/autograd.py).

Checks:
  * the gradients equal torch.autograd through torch.matmul (cuBLAS, FP64) to
    <= 1e-12 relative;
  * central finite differences, h = 1e-6, on 16 random unit-norm directions
    and 32 single coordinates (stepped along the gradient component, so real
    and imaginary parts both enter) per operand agree with Re<grad, dX> to
    <= 1e-6 relative (dX = (X + hV) - (X - hV) as evaluated), the difference
    quotient being evaluated in the cancellation-free form of the quadratic
    loss (see _fd_check); the plain two-evaluation difference, whose accuracy
    at h = 1e-6 is bounded by the FP64 rounding of the forwards, agrees to
    <= 2e-3;
  * the plain two-evaluation difference over a range of h (1e-6 ... 1e-2):
    for this quadratic loss the central difference has no truncation error,
    so its discrepancy is rounding alone and falls as 1/h, reaching <= 1e-6
    at h >= 1e-3 (the measured table is printed and written to
    fd_vs_h.json in the pytest temporary directory);
  * the Ozaki path's gradient equals the FP64 DMMA path's.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M = N = 512
K = 100000
H = 1e-6


@pytest.fixture(scope="module")
def setup():
    import torch
    import spla_b200 as spla
    g = torch.Generator(device="cuda")
    g.manual_seed(20250005)
    s = (1.0 / (2 * K)) ** 0.5
    A = torch.randn((M, K), dtype=torch.complex128, device="cuda", generator=g) * s
    B = torch.randn((N, K), dtype=torch.complex128, device="cuda", generator=g) * s
    ctx = spla.Context(spla.PU_GPU)
    ctx.set_fp64_path(spla.PATH_DMMA)
    return torch, spla, A, B, ctx


def loss_exact(C):
    """m + sum |C|^2 - 2 Re tr C, exactly rounded sum on the host."""
    c = C.detach().cpu().numpy()
    terms = np.concatenate([(c.real ** 2).ravel(), (c.imag ** 2).ravel(),
                            -2.0 * np.diag(c).real])
    return M + math.fsum(terms.tolist())


def grads(torch, spla, A, B, ctx):
    from spla_b200.autograd import ssb_autograd
    Ar = A.clone().requires_grad_(True)
    Br = B.clone().requires_grad_(True)
    C = ssb_autograd(Ar, Br, ctx)
    eye = torch.eye(M, N, dtype=C.dtype, device=C.device)
    L = (C - eye).abs().pow(2).sum()
    L.backward()
    return Ar.grad.detach(), Br.grad.detach()


def test_gradient_matches_torch_autograd(setup):
    torch, spla, A, B, ctx = setup
    gA, gB = grads(torch, spla, A, B, ctx)
    Ar = A.clone().requires_grad_(True)
    Br = B.clone().requires_grad_(True)
    C = Ar.conj() @ Br.T
    eye = torch.eye(M, N, dtype=C.dtype, device=C.device)
    ((C - eye).abs().pow(2).sum()).backward()
    for got, ref in ((gA, Ar.grad), (gB, Br.grad)):
        rel = float((got - ref).norm() / ref.norm())
        assert rel <= 1e-12, rel


def _fd_check(torch, spla, A, B, ctx, which, gA, gB):
    """Central differences at h = 1e-6 along V, compared with Re<grad, dX>,
    dX = X+ - X- the realised step (X+- = X +- hV as rounded).

    For the quadratic loss, L(X+) - L(X-) = Re<C+ + C- - 2I, C+ - C->
    exactly, and C+ - C- = forward(dX) by linearity. Two estimates:
      stable: that identity with three forward evaluations - no cancellation;
      raw:    L(X+) - L(X-) from two forward evaluations and exact host sums.
    At h = 1e-6 the raw form is limited by the FP64 rounding of the two
    forwards (~1e-5 relative here; the same holds for torch.matmul through
    cuBLAS, which gives the identical value). Returns the worst relative
    discrepancy of each estimate."""
    from spla_b200.autograd import ssb
    rng = np.random.default_rng(17 if which == "A" else 18)
    X = A if which == "A" else B
    grad = gA if which == "A" else gB
    eye = torch.eye(M, N, dtype=X.dtype, device=X.device)
    worst_stable = worst_raw = 0.0
    dirs = []
    for _ in range(16):
        V = torch.from_numpy(rng.standard_normal(X.shape) + 1j * rng.standard_normal(X.shape)).to(
            X.device)
        dirs.append(V / V.norm())
    for _ in range(32):
        idx = (int(rng.integers(X.shape[0])), int(rng.integers(X.shape[1])))
        V = torch.zeros_like(X)
        gi = complex(grad[idx].item())
        V[idx] = gi / abs(gi)  # unit step along the gradient component: real and imaginary parts
        dirs.append(V)

    def fwd(Xv):
        return ssb(Xv, B, ctx) if which == "A" else ssb(A, Xv, ctx)

    for V in dirs:
        Xp, Xm = X + H * V, X - H * V
        dX = Xp - Xm
        Cp, Cm, dC = fwd(Xp), fwd(Xm), fwd(dX)
        an = float((grad.conj() * dX).sum().real)
        stable = float(((Cp + Cm - 2 * eye).conj() * dC).sum().real)
        raw = loss_exact(Cp) - loss_exact(Cm)
        worst_stable = max(worst_stable, abs(stable - an) / abs(an))
        worst_raw = max(worst_raw, abs(raw - an) / abs(an))
    return worst_stable, worst_raw


@pytest.mark.parametrize("which", ["A", "B"])
def test_finite_differences(setup, which):
    torch, spla, A, B, ctx = setup
    gA, gB = grads(torch, spla, A, B, ctx)
    stable, raw = _fd_check(torch, spla, A, B, ctx, which, gA, gB)
    assert stable <= 1e-6, stable
    assert raw <= 2e-3, raw


def test_plain_central_difference_vs_h(setup, tmp_path):
    """(L(X + hV) - L(X - hV)) / 2 with two forwards only, against Re<grad, dX>,
    for h from 1e-6 to 1e-2 on 8 random unit directions of A: the worst
    relative discrepancy times h stays about constant (rounding of the
    forwards, no truncation term), and the plain form meets 1e-6 once h is
    large enough for the rounding to be below it."""
    import json
    torch, spla, A, B, ctx = setup
    from spla_b200.autograd import ssb
    gA, _ = grads(torch, spla, A, B, ctx)
    rng = np.random.default_rng(19)
    dirs = []
    for _ in range(8):
        V = torch.from_numpy(rng.standard_normal(A.shape) + 1j * rng.standard_normal(A.shape)).to(
            A.device)
        dirs.append(V / V.norm())
    table = {}
    for h in (1e-6, 1e-5, 1e-4, 1e-3, 1e-2):
        worst = 0.0
        for V in dirs:
            Xp, Xm = A + h * V, A - h * V
            an = float((gA.conj() * (Xp - Xm)).sum().real)
            raw = loss_exact(ssb(Xp, B, ctx)) - loss_exact(ssb(Xm, B, ctx))
            worst = max(worst, abs(raw - an) / abs(an))
        table[h] = worst
    print("plain central difference, worst relative discrepancy by h:", table)
    (tmp_path / "fd_vs_h.json").write_text(json.dumps({str(h): v for h, v in table.items()}))
    assert table[1e-6] <= 2e-3
    assert table[1e-3] <= 1e-6 and table[1e-2] <= 1e-6, table
    # rounding-limited: the discrepancy falls with h (within a factor for noise)
    assert table[1e-2] < table[1e-6] / 100, table


def test_ozaki_forward_gradient_matches_dmma(setup):
    torch, spla, A, B, ctx = setup
    gA, gB = grads(torch, spla, A, B, ctx)
    ctx_o = spla.Context(spla.PU_GPU)
    ctx_o.set_fp64_path(spla.PATH_OZAKI)
    oA, oB = grads(torch, spla, A, B, ctx_o)
    for got, ref in ((oA, gA), (oB, gB)):
        rel = float((got - ref).norm() / ref.norm())
        assert rel <= 1e-13, rel
