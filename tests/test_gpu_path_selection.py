"""AUTO path resolution (splab_gemm_path): the measured cost model picks DMMA
for small contractions, Ozaki for large FP64 ones, 3xTF32 for mid-size float
ones; explicit paths resolve to themselves where supported and to DMMA
otherwise; resolving, sizing and running agree (the workspace of the resolved
path is what a run with AUTO needs)."""
import numpy as np
import pytest

import spla_b200 as spla

pytestmark = pytest.mark.gpu

C64, R64, C32, R32 = 3, 1, 2, 0
DMMA, OZAKI, TF3 = spla.PATH_DMMA, spla.PATH_OZAKI, spla.PATH_TF32X3


@pytest.mark.parametrize("dt,m,k,want", [
    (C64, 128, 8192, DMMA), (C64, 256, 32768, DMMA), (C64, 1024, 250000, OZAKI),
    (C64, 2048, 8192, OZAKI), (R64, 256, 8192, DMMA), (R64, 2048, 8192, OZAKI),
    (C32, 128, 8192, DMMA), (C32, 256, 32768, TF3), (C32, 2048, 8192, OZAKI),
    (R32, 512, 65536, TF3)])
def test_auto_resolution(dt, m, k, want):
    opA = 2 if dt in (C64, C32) else 1
    assert spla.lib().splab_gemm_path(dt, spla.PATH_AUTO, opA, 0, m, m, k) == want


def test_explicit_paths():
    L = spla.lib()
    assert L.splab_gemm_path(C64, OZAKI, 2, 0, 64, 64, 100) == OZAKI
    assert L.splab_gemm_path(C64, TF3, 2, 0, 4096, 4096, 100000) == DMMA  # double: no 3xTF32
    # any op pair on the tensor-core paths (k-major copies of op(A) = N / op(B) != N)
    assert L.splab_gemm_path(C32, TF3, 0, 0, 512, 512, 4096) == TF3       # op(A) = N
    assert L.splab_gemm_path(C64, OZAKI, 0, 1, 64, 64, 100) == OZAKI      # op(B) = T
    assert L.splab_gemm_path(C32, TF3, 2, 2, 64, 64, 100) == TF3          # op(B) = C
    # op(A) = N on Ozaki (A copied k-major first): the subspace rotation shape
    assert L.splab_gemm_path(C64, spla.PATH_AUTO, 0, 0, 200000, 2048, 2048) == OZAKI
    assert L.splab_gemm_path(C64, spla.PATH_AUTO, 0, 0, 4096, 4096, 100000) == OZAKI


def test_auto_workspace_matches_run():
    import torch
    m = n = 512
    k = 16384
    path = spla.lib().splab_gemm_path(C64, spla.PATH_AUTO, 2, 0, m, n, k)
    ws_auto = spla.splab_gemm_workspace_size("complex128", spla.PATH_AUTO, 2, 0, m, n, k)
    assert ws_auto == spla.splab_gemm_workspace_size("complex128", path, 2, 0, m, n, k)
    A = torch.randn(m * k, dtype=torch.complex128, device="cuda")
    B = torch.randn(n * k, dtype=torch.complex128, device="cuda")
    C = torch.zeros(m * n, dtype=torch.complex128, device="cuda")
    ws = torch.empty(max(1, ws_auto), dtype=torch.uint8, device="cuda")
    assert spla.splab_gemm("complex128", spla.PATH_AUTO, 2, 0, m, n, k, 1.0, A, k, B, k, 0.0, C,
                           m, workspace=ws, workspace_bytes=ws_auto) == 0
    torch.cuda.synchronize()
    ref = (A.view(m, k).conj() @ B.view(n, k).T).T.reshape(-1)
    assert float((C - ref).norm() / ref.norm()) <= 1e-13
