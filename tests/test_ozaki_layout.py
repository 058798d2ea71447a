"""Workspace layout of the Ozaki path, checked on the CPU through the kernel C
ABI's sizing call (no device needed): complex products keep three residue
planes per modulus and operand (re, im and their sum), real ones a single
plane; the residues of C are bytes when the contraction is one k-chunk (at
most 124928 residue bytes per row) and int32 sums beyond; op(A) = N and
op(B) = T, C are read in place (no k-major copy: only the partial sums of the
k-sliced row norms); the modulus count follows the dtype default or the knob."""
import spla_b200 as spla

OZ = spla.PATH_OZAKI
SLACK = 1 << 20  # row exponents, status word, tile list and 256-byte alignment


def ws(dtype, opA, m, n, k, moduli=0, opB=0):
    return spla.splab_gemm_workspace_size(dtype, OZ, opA, opB, m, n, k, moduli)


def kp(k):
    return (k + 127) // 128 * 128


def test_complex_three_planes_per_modulus():
    m, n, k = 1024, 768, 50000
    planes = 15 * 3 * (m + n) * kp(k)  # residues of A and B
    r8 = 15 * 3 * n * m                # one k-chunk: byte residues of the products
    assert planes + r8 <= ws("complex128", 2, m, n, k) <= planes + r8 + SLACK


def test_real_one_plane_per_modulus():
    m, n, k = 1024, 768, 50000
    planes = 15 * (m + n) * kp(k)
    r8 = 15 * n * m
    assert planes + r8 <= ws("float64", 1, m, n, k) <= planes + r8 + SLACK


def test_int32_sums_beyond_one_chunk():
    m = n = 512
    one = ws("complex128", 2, m, n, 124928)  # 976 blocks of 128 bytes: one chunk
    two = ws("complex128", 2, m, n, 124929)  # 977 blocks: two chunks
    plane_growth = 15 * 3 * (m + n) * 128    # one more block per residue row
    r_growth = 15 * 3 * n * m * 3            # product residues: bytes -> int32
    assert abs((two - one) - (plane_growth + r_growth)) <= 4096


def norm_slices(rows, k):
    """k-slices of the in-place row norms (about 2^18 threads, >= 512 elements each)"""
    if rows >= 65536 or k <= 512:
        return 1
    return max(1, min(-(-(1 << 18) // rows), 4096, -(-k // 512)))


def partials(rows, k):
    s = norm_slices(rows, k)
    return s * rows * 12 if s > 1 else 0  # a double and an int per row and slice


def test_in_place_operands_need_no_copy():
    m, n, k = 2000, 256, 3000
    diff = ws("complex128", 0, m, n, k) - ws("complex128", 1, m, n, k)
    assert abs(diff - partials(m, k)) <= 512  # op(A) = N: no copy of A (96 MB)
    for opB in (1, 2):
        diff = ws("complex128", 1, m, n, k, opB=opB) - ws("complex128", 1, m, n, k)
        assert abs(diff - partials(n, k)) <= 512
    # many rows: the norms are not sliced
    assert ws("complex128", 0, 70000, 64, 2048) - ws("complex128", 1, 70000, 64, 2048) == 0
    # a few rows and a long k: at most 4096 slices (the launch grid's y extent)
    m, k = 4, 4_000_000
    diff = ws("float64", 0, m, 8, k) - ws("float64", 1, m, 8, k)
    assert abs(diff - partials(m, k)) <= 512 and norm_slices(m, k) == 4096


def test_modulus_count():
    m = n = 512
    k = 20000
    per_modulus = 3 * (m + n) * kp(k) + 3 * n * m
    c64, c128 = ws("complex64", 2, m, n, k), ws("complex128", 2, m, n, k)
    assert abs((c128 - c64) - 6 * per_modulus) <= SLACK  # 15 vs 9 moduli
    c12 = ws("complex128", 2, m, n, k, moduli=12)
    assert abs((c128 - c12) - 3 * per_modulus) <= SLACK
