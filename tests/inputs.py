"""Seeded input generators shared by the golden-fixture script, the tests and
the benchmark. Matrices are flat column-major numpy buffers of
`ld * cols` elements (ld >= rows); padding entries are filled too, so that
"padding untouched" checks see real data.

Distributions (named as in the benchmark configurations):
  uniform100 : entries (and for complex, real and imaginary parts) U[0, 100),
               the reference tests' distribution (tests/test_gemm.cpp:46-60)
  uniform11  : U[-1, 1]
  gauss_k    : Gaussian scaled by 1/sqrt(k); complex entries have real and
               imaginary parts N(0, 1/(2k)) so that E|z|^2 = 1/k
"""
from __future__ import annotations

import numpy as np


def buffer(dtype, ld, cols, seed, dist="uniform100", k=1):
    dtype = np.dtype(dtype)
    rng = np.random.default_rng(seed)
    n = max(0, ld * cols)
    cplx = dtype.kind == "c"
    real_dt = np.float32 if dtype in (np.float32, np.complex64) else np.float64

    def draw(size):
        if dist == "uniform100":
            return rng.random(size) * 100.0
        if dist == "uniform11":
            return rng.uniform(-1.0, 1.0, size)
        if dist == "gauss_k":
            s = 1.0 / np.sqrt((2.0 if cplx else 1.0) * max(1, k))
            return rng.standard_normal(size) * s
        raise ValueError(dist)

    if cplx:
        v = draw(2 * n).astype(real_dt).view(dtype)
    else:
        v = draw(n).astype(real_dt)
    return np.ascontiguousarray(v.astype(dtype))


def col_major_view(buf, rows, cols, ld):
    """(rows x cols) strided view of a flat column-major buffer."""
    return buf[: ld * cols].reshape(cols, ld)[:, :rows].T if rows and cols else buf[:0].reshape(0, 0)


def sample_indices(size, count, seed):
    if size <= count:
        return np.arange(size)
    return np.sort(np.random.default_rng(seed).choice(size, count, replace=False))
