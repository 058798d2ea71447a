"""CPU check of the residue arithmetic of the Ozaki slicer (oz_slice):
digits of the scaled integer x, their sum s = sum_j c_j d_j with c_j =
base^j mod p centred (as the host sets them), and FP32 residues through a
1.5 * 2^23 magic constant. Three digit forms, as the slicer picks them:
  * double, default modulus count: four balanced base-2^15 digits of
    |x| < 2^58 (d0, d2 in [-2^14, 2^14), d1 in [-2^14, 2^14], d3 in
    [-2^13, 2^13]); the remainder is formed first, then biased;
  * double, 16 moduli: five base-2^13 digits of |x| < 2^62 (d0, d2, d3 in
    [0, 2^13), d1 in [-2^12, 2^12], d4 in [-2^10, 2^10]);
  * float, default count: three base-2^13 digits of |x| < 2^38 (d0 in
    [0, 2^13), d1, d2 in [-2^12 - 1, 2^12 + 1]);
the last two add the bias to s before the remainder, so s + M must be exact
(|s| < 2^22). For every odd modulus of the form and EVERY digit sum its
digits can give, the quotient q = fl32(s * fl32(1/p) + M) - M, evaluated in
exact integer arithmetic with round-to-nearest-even as the FP32 FMA does,
must be the nearest integer to s / p, so that r = s - q p is the centred
residue with |r| <= 127 (one signed byte). The same is checked for the
third-plane step, t = r(re) +- r(im). The moduli and their default counts are
read from the kernel header, so the check follows the code."""
import re
from pathlib import Path

import numpy as np
import pytest

HDR = Path(__file__).resolve().parent.parent / "spla_b200" / "csrc" / "kernels" / "ozaki_crt.cuh"
M = 12582912  # 1.5 * 2^23


def _moduli(count_name):
    text = HDR.read_text()
    table = re.search(r"kModuli\[kMaxModuli\]\s*=\s*\{([^}]*)\}", text).group(1)
    moduli = [int(v) for v in table.replace("\n", " ").split(",") if v.strip()]
    n = int(re.search(count_name + r"\s*=\s*(\d+)", text).group(1))
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


# (moduli, digit base, largest |d_j| per digit, bias added before the remainder)
FORMS = {
    "double_4x15": (lambda: _moduli("kDefaultModuli"), 1 << 15,
                    [1 << 14, 1 << 14, 1 << 14, 1 << 13], False),
    "double_5x13": (lambda: _moduli("kMaxUsableModuli"), 1 << 13,
                    [(1 << 13) - 1, 1 << 12, (1 << 13) - 1, (1 << 13) - 1, 1 << 10], True),
    "float_3x13": (lambda: _moduli("kDefaultModuliFloat"), 1 << 13,
                   [(1 << 13) - 1, (1 << 12) + 1, (1 << 12) + 1], True),
}


@pytest.mark.parametrize("form", list(FORMS))
def test_digit_sums_give_centred_byte_residues(form):
    moduli_of, base, dmax, bias_first = FORMS[form]
    checked = 0
    for p in moduli_of():
        if p == 256:  # residue = low byte of the lowest digit, no quotient step
            continue
        c = [1] + [_centred(pow(base, j, p), p) for j in range(1, len(dmax))]
        smax = sum(abs(cj) * dj for cj, dj in zip(c, dmax))
        assert smax < (1 << 23), (p, smax)  # FMA chain exact; quotient input in range
        if bias_first:
            assert smax < (1 << 22), (p, smax)  # s + M exact
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
    assert checked > 1_000_000
