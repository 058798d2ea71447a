"""CPU check of the residue arithmetic of the Ozaki slicer (oz_slice, the
default complex-double form: four balanced base-2^15 digits, FP32 residues
through a 1.5 * 2^23 magic constant).

For every default odd modulus p and EVERY digit sum s the four digits of a
scaled integer |x| < 2^58 can give (d0, d2 in [-2^14, 2^14), d1 in
[-2^14, 2^14], d3 in [-2^13, 2^13]; s = d0 + c1 d1 + c2 d2 + c3 d3 with
c_j = 2^(15 j) mod p centred, as the host sets them), the quotient step
q = fl32(s * fl32(1/p) + M) - M, evaluated here in exact integer arithmetic
with round-to-nearest-even as the FP32 FMA does, must give the nearest
integer to s / p, so that the remainder r = s - q p is the centred residue
with |r| <= 127 (one signed byte). The digit sums themselves stay below 2^24
(exact in FP32). The same is checked for the third-plane step, t = r(re) +-
r(im) with |t| <= 254. The moduli and their default count are read from the
kernel header, so the check follows the code."""
import re
from pathlib import Path

import numpy as np

HDR = Path(__file__).resolve().parent.parent / "spla_b200" / "csrc" / "kernels" / "ozaki_crt.cuh"
M = 12582912  # 1.5 * 2^23


def _moduli():
    text = HDR.read_text()
    table = re.search(r"kModuli\[kMaxModuli\]\s*=\s*\{([^}]*)\}", text).group(1)
    moduli = [int(v) for v in table.replace("\n", " ").split(",") if v.strip()]
    n = int(re.search(r"kDefaultModuli\s*=\s*(\d+)", text).group(1))
    return moduli[:n]


def _centred(w, p):
    return w - p if w > p // 2 else w


def _quotient(s, p):
    """fl32(s * fl32(1/p) + M) - M for int64 s, exactly (|s| < 2^23)."""
    ip = np.float32(1.0) / np.float32(p)
    frac, exp = np.frexp(np.float64(ip))  # ip = frac 2^exp, frac in [0.5, 1)
    mant = int(frac * (1 << 24))          # ip = mant 2^(exp - 24), mant < 2^24
    sh = 24 - int(exp)
    assert float(mant) * 2.0 ** (exp - 24) == float(ip)
    N = s * mant + (M << sh)              # (s ip + M) 2^sh, exact in int64
    fl = N >> sh
    rem = N - (fl << sh)
    half = 1 << (sh - 1)
    up = (rem > half) | ((rem == half) & (fl % 2 == 1))
    return fl + up.astype(np.int64) - M


def test_digit_sums_give_centred_byte_residues():
    checked = 0
    for p in _moduli():
        if p == 256:  # residue = low byte of the lowest digit, no quotient step
            continue
        c = [_centred(pow(1 << 15, j, p), p) for j in (1, 2, 3)]
        smax = (1 << 14) + abs(c[0]) * (1 << 14) + abs(c[1]) * (1 << 14) + abs(c[2]) * (1 << 13)
        assert smax < (1 << 23), (p, smax)  # FMA chain exact; quotient input in range
        for lo in range(-smax, smax + 1, 1 << 22):
            s = np.arange(lo, min(lo + (1 << 22), smax + 1), dtype=np.int64)
            q = _quotient(s, p)
            r = s - q * p
            assert np.all(np.abs(r) <= 127), p
            assert np.all(2 * np.abs(r) <= p), p          # the nearest quotient
            assert np.all((r - s) % p == 0), p
            checked += s.size
        # the third plane: t = r(re) + s_sum r(im), |t| <= 2 (p - 1) / 2
        h = (p - 1) // 2
        t = np.arange(-2 * h, 2 * h + 1, dtype=np.int64)
        r = t - _quotient(t, p) * p
        assert np.all(2 * np.abs(r) <= p) and np.all((r - t) % p == 0), p
    assert checked > 50_000_000
