"""Load the golden fixtures (tests/golden/) and rebuild their seeded inputs."""
from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

from inputs import buffer

GOLDEN = Path(__file__).resolve().parent / "golden"
DT = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}


@lru_cache(maxsize=None)
def load(name):
    cases = json.loads((GOLDEN / f"{name}.json").read_text())
    arrays = dict(np.load(GOLDEN / f"{name}.npz"))
    return cases, arrays


def expected(name, case):
    _, arrays = load(name)
    return arrays[f"c{case['id']}_idx"], arrays[f"c{case['id']}_val"]


def scalar(v, dt):
    if isinstance(v, list):
        return complex(v[0], v[1]) if np.dtype(dt).kind == "c" else v[0]
    return v


def gemm_inputs(c):
    dt = DT[c["dtype"]]
    A = buffer(dt, c["lda"], c["k"] if c["opA"] == 0 else c["m"], c["seed"])
    B = buffer(dt, c["ldb"], c["n"] if c["opB"] == 0 else c["k"], c["seed"] + 50000)
    C = buffer(dt, c["ldc"], c["n"], c["seed"] + 90000)
    return dt, A, B, C


def ssb_inputs(c):
    dt = DT[c["dtype"]]
    A = buffer(dt, c["lda"], c["m"], c["seed"])
    B = buffer(dt, c["ldb"], c["n"], c["seed"] + 50000)
    C = buffer(dt, c["ldc"], c["n"] + c["co"], c["seed"] + 90000)
    return dt, A, B, C


def sbs_inputs(c):
    dt = DT[c["dtype"]]
    A = buffer(dt, c["lda"], c["k"], c["seed"])
    B = buffer(dt, c["ldb"], c["n"] + c["bco"], c["seed"] + 50000)
    C = buffer(dt, c["ldc"], c["n"], c["seed"] + 90000)
    return dt, A, B, C


def tolerance(dt, k):
    """Relative tolerance of a parity comparison against the reference BLAS output.

    double: the reference's own test bar is abs 1e-6 on values up to ~1e7
    (tests/test_gemm.cpp:80-81); we require |x - ref| <= 1e-13 * scale, with
    scale the magnitude of the largest term. float: 1e-6 relative.
    """
    return 1e-6 if np.dtype(dt) in (np.float32, np.complex64) else 1e-13


def fill_mask(c, idx):
    """Boolean mask over C-buffer indices `idx`: True where the element is in the
    computed part of C (inside the m x n block and, for a fill mode, in the
    triangle incl. diagonal, in the global coordinates of the distributed C)."""
    ldc, ro, co, m, n = c["ldc"], c["ro"], c["co"], c["m"], c["n"]
    r, col = idx % ldc, idx // ldc
    inside = (r >= ro) & (r < ro + m) & (col >= co) & (col < co + n)
    if c.get("fill", 0) == 1:
        inside &= col >= r  # upper: global col >= global row
    elif c.get("fill", 0) == 2:
        inside &= r >= col
    return inside
