// Chinese-remainder constants and reconstruction of the Ozaki scheme II path
// (host and device code): exact integer arithmetic on 32-bit limbs up to the
// final conversion to double, and the division-free reduction of the INT8
// GEMM's int32 sums modulo each modulus.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

namespace splab {
namespace oz {

inline constexpr int kMaxModuli = 20;  // table size
// The product of the moduli must fit 128 bits: at most 16 (2^124.4).
inline constexpr int kMaxUsableModuli = 16;
// Pairwise coprime moduli <= 256, largest first (256 = 2^8, 255 = 3*5*17,
// 253 = 11*23, 247 = 13*19, 217 = 7*31, the rest prime).
inline constexpr int kModuli[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                     223, 217, 211, 199, 197, 193, 191, 181, 179, 173};
inline constexpr int kDefaultModuli = 15;       // double: Q = 57
inline constexpr int kDefaultModuliFloat = 9;   // float: Q = 34

struct Crt {
  int n;
  int p[kMaxModuli];
  double inv_p[kMaxModuli];
  unsigned long long w_lo[kMaxModuli], w_hi[kMaxModuli];  // CRT weights W_t < P
  unsigned long long P_lo, P_hi;
  double P_d;
  int q_bits;  // Q: scaled rows have 2-norm < 2^Q
};

// --------------------------------------------------------------------------
// host: CRT constants

inline Crt make_crt(int n) {
  Crt c{};
  c.n = n;
  unsigned __int128 P = 1;
  for (int t = 0; t < n; ++t) P *= (unsigned __int128)kModuli[t];
  for (int t = 0; t < n; ++t) {
    const int p = kModuli[t];
    c.p[t] = p;
    c.inv_p[t] = 1.0 / double(p);
    const unsigned __int128 Mt = P / (unsigned __int128)p;
    const int mt_mod = int(Mt % (unsigned __int128)p);
    int y = 1;
    while ((mt_mod * y) % p != 1) ++y;  // modular inverse, p <= 256
    const unsigned __int128 W = Mt * (unsigned __int128)y;  // < P since y < p
    c.w_lo[t] = (unsigned long long)W;
    c.w_hi[t] = (unsigned long long)(W >> 64);
  }
  c.P_lo = (unsigned long long)P;
  c.P_hi = (unsigned long long)(P >> 64);
  c.P_d = double(c.P_hi) * 18446744073709551616.0 + double(c.P_lo);
  // |X| <= (2^Q + sqrt(K)/2)^2 must stay below P/2: Q = floor((log2 P - 2) / 2).
  const double lp = std::log2(c.P_d);
  c.q_bits = int(std::floor((lp - 2.0) / 2.0));
  return c;
}

// v mod p in [0, p) for any int32 v and 2 <= p <= 256 without a division:
// v = hi * 2^16 + lo, t = hi * (2^16 mod p) + lo = v (mod p) with |t| < 2^24,
// x = t + off (off a multiple of p, >= 2^24) in [0, 2^26), and
// floor(x / p) = floor(x * M / 2^34) with M = ceil(2^34 / p): the product
// overestimates x / p by less than x / 2^34 < 2^-8 <= 1 / p, which cannot
// reach the next integer.
struct ModMagic {
  int c16;     // 2^16 mod p
  int off;     // p * ceil(2^24 / p)
  unsigned M;  // ceil(2^34 / p) < 2^27
};

inline ModMagic make_mod_magic(int p) {
  ModMagic mm;
  mm.c16 = 65536 % p;
  mm.off = p * (((1 << 24) + p - 1) / p);
  mm.M = unsigned(((1ull << 34) + unsigned(p) - 1) / unsigned(p));
  return mm;
}

__host__ __device__ __forceinline__ int mod_residue(int v, int p, int c16, int off, unsigned M) {
  const int hi = v >> 16;  // arithmetic shift
  const int lo = v & 0xFFFF;
  const unsigned x = unsigned(hi * c16 + lo + off);
#ifdef __CUDA_ARCH__
  const unsigned q = __umulhi(x, M) >> 2;
#else
  const unsigned q = unsigned((unsigned long long)x * M >> 34);
#endif
  return int(x - q * unsigned(p));
}

struct ReconParams {
  int n;
  int p[kMaxModuli];
  int off24[kMaxModuli];      // p * ceil(2^24 / p): a multiple of p above any int32 residue sum
  unsigned w[kMaxModuli][4];  // CRT weights W_t < P as 32-bit limbs, least significant first
  unsigned P[4];              // P as 32-bit limbs
  double inv_P32;             // 2^32 / P
  int conj;                   // complex products: A^H B (1) or A^T B / A B (0)
};

// Residues of Re and Im of a complex product from the residues of the three
// real products P0 = re(a) re(b), P1 = im(a) im(b), P2 = (re(a) + s im(a))
// (re(b) + im(b)) with s = -1 for A^H B (conj(a) b: Re = P0 + P1,
// Im = P2 - P0 + P1) and s = +1 otherwise (Re = P0 - P1, Im = P2 - P0 - P1).
// off is a multiple of p not below any r (p for bytes, off24 for int32 sums),
// so the results are non-negative and below 3 off.
__host__ __device__ __forceinline__ void combine3(int r0, int r1, int r2, int off, int conj,
                                                  int& re, int& im) {
  if (conj) {
    re = r0 + r1;
    im = r2 + r1 + (off - r0);
  } else {
    re = r0 + (off - r1);
    im = r2 + (off - r0) + (off - r1);
  }
}

inline ReconParams make_recon(const Crt& c) {
  ReconParams rp{};
  rp.n = c.n;
  for (int t = 0; t < c.n; ++t) {
    rp.p[t] = c.p[t];
    rp.off24[t] = c.p[t] * (((1 << 24) + c.p[t] - 1) / c.p[t]);
    const unsigned long long lo = c.w_lo[t], hi = c.w_hi[t];
    rp.w[t][0] = unsigned(lo);
    rp.w[t][1] = unsigned(lo >> 32);
    rp.w[t][2] = unsigned(hi);
    rp.w[t][3] = unsigned(hi >> 32);
  }
  rp.P[0] = unsigned(c.P_lo);
  rp.P[1] = unsigned(c.P_lo >> 32);
  rp.P[2] = unsigned(c.P_hi);
  rp.P[3] = unsigned(c.P_hi >> 32);
  rp.inv_P32 = 4294967296.0 / c.P_d;
  return rp;
}

// Exact conversions to double of integers below 2^32 and 2^52: the integer
// is placed in the mantissa of 2^52 and 2^52 subtracted (one FP64 add instead
// of an integer-to-float conversion).
__host__ __device__ __forceinline__ double u32_to_double(unsigned x) {
#ifdef __CUDA_ARCH__
  return __hiloint2double(0x43300000, int(x)) - 4503599627370496.0;
#else
  return double(x);
#endif
}
// The same for a signed integer of magnitude below 2^31 (offset by 2^31).
__host__ __device__ __forceinline__ double i32_to_double(int x) {
#ifdef __CUDA_ARCH__
  return __hiloint2double(0x43300000, x ^ int(0x80000000u)) - 4503601774854144.0;
#else
  return double(x);
#endif
}
__host__ __device__ __forceinline__ double u52_to_double(unsigned long long x) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)(x | 0x4330000000000000ull)) - 4503599627370496.0;
#else
  return double(x);
#endif
}

// X = (sum_t W_t r_t) mod P as the representative of smallest magnitude,
// converted to double (within 1.5 units in the last place), for values with
// |X| <= P/4: the row scaling of the Ozaki path bounds every element of the
// scaled product by (2^Q + sqrt(K)/2)^2 with 2^(2Q) <= P/4.
//
// S = sum_t W_t r_t is accumulated per 32-bit limb of W_t (one 32x32->64
// multiply-add per limb and modulus, no carries: r_t < 2^26 and at most 16
// terms keep each limb sum below 2^62). S / P lies within 1/4 + 2^-37 of the
// integer q = round(S / P), and the estimate S * (2^32 / P) from the top
// three limb sums in double is off by less than 2^-20, so rounding it gives q
// exactly. X = S - qP is formed limb by limb in signed 64-bit arithmetic,
// carried into 32-bit limbs x0..x2 and a small signed top c, and converted by
// Horner's rule in FP64 (exact while the partial value is below 2^53; after
// that each of at most three steps rounds once, relative to a partial value
// no larger than about |X|).
//
// N: number of moduli (0: rp.n at run time). BYTES: residues below 2^10 (the
// limb sums are then below 2^46 and convert exactly by the mantissa method).
//
// crt_from_limbs: the same from S given as limb sums, S = l0 + l1 2^32 +
// l2 2^64 + l3 2^96 with every l below 2^62 (below 2^52 with BYTES), and
// S / P below 2^14.
template <bool BYTES>
__host__ __device__ __forceinline__ double crt_from_limbs(unsigned long long l0,
                                                          unsigned long long l1,
                                                          unsigned long long l2,
                                                          unsigned long long l3,
                                                          const ReconParams& rp) {
  // q = round(S / P) from (l1 + l2 2^32 + l3 2^64) * 2^32 / P
  double s1, s2, s3;
  if (BYTES) {
    s1 = u52_to_double(l1);
    s2 = u52_to_double(l2);
    s3 = u52_to_double(l3);
  } else {
    s1 = double(l1);
    s2 = double(l2);
    s3 = double(l3);
  }
  const double sh = fma(s3, 18446744073709551616.0, fma(s2, 4294967296.0, s1));
  const double qr = fma(sh, rp.inv_P32, 6755399441055744.0);  // 1.5 * 2^52: rounds to integer
#ifdef __CUDA_ARCH__
  const unsigned q = unsigned(__double2loint(qr));
#else
  const unsigned q = unsigned((unsigned long long)(qr - 6755399441055744.0));
#endif
  // X = S - qP, limb by limb (each difference lies in (-2^62, 2^62)), carried
  const unsigned long long qq = q;
  long long c = (long long)(l0 - qq * rp.P[0]);
  const unsigned x0 = unsigned(c);
  c = (c >> 32) + (long long)(l1 - qq * rp.P[1]);
  const unsigned x1 = unsigned(c);
  c = (c >> 32) + (long long)(l2 - qq * rp.P[2]);
  const unsigned x2 = unsigned(c);
  c = (c >> 32) + (long long)(l3 - qq * rp.P[3]);  // |c| < 2^22
  double v = fma(i32_to_double(int(c)), 4294967296.0, u32_to_double(x2));
  v = fma(v, 4294967296.0, u32_to_double(x1));
  return fma(v, 4294967296.0, u32_to_double(x0));
}

template <int N, bool BYTES>
__host__ __device__ __forceinline__ double crt_value(const int* r, const ReconParams& rp) {
  unsigned long long l0 = 0, l1 = 0, l2 = 0, l3 = 0;
#pragma unroll
  for (int t = 0; t < (N > 0 ? N : kMaxUsableModuli); ++t) {
    if (N == 0 && t >= rp.n) break;
    const unsigned rt = unsigned(r[t]);
    l0 += (unsigned long long)rt * rp.w[t][0];
    l1 += (unsigned long long)rt * rp.w[t][1];
    l2 += (unsigned long long)rt * rp.w[t][2];
    l3 += (unsigned long long)rt * rp.w[t][3];
  }
  return crt_from_limbs<BYTES>(l0, l1, l2, l3, rp);
}

}  // namespace oz
}  // namespace splab
