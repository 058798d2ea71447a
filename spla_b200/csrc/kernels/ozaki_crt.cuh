// Chinese-remainder constants and reconstruction of the Ozaki scheme II path
// (host and device code). The reconstruction is exact integer arithmetic on
// 64-bit limbs; see ozaki.cu for the method.
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

struct ReconParams {
  int n;
  int p[kMaxModuli];
  unsigned long long w_lo[kMaxModuli], w_hi[kMaxModuli];
  unsigned long long P_lo, P_hi;
  double P_d, inv_P;
};

inline ReconParams make_recon(const Crt& c) {
  ReconParams rp{};
  rp.n = c.n;
  for (int t = 0; t < c.n; ++t) {
    rp.p[t] = c.p[t];
    rp.w_lo[t] = c.w_lo[t];
    rp.w_hi[t] = c.w_hi[t];
  }
  rp.P_lo = c.P_lo;
  rp.P_hi = c.P_hi;
  rp.P_d = c.P_d;
  rp.inv_P = 1.0 / c.P_d;
  return rp;
}

__host__ __device__ __forceinline__ unsigned long long mulhi64(unsigned long long a,
                                                               unsigned long long b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (unsigned long long)(((unsigned __int128)a * b) >> 64);
#endif
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

// Correctly rounded conversion of the signed 128-bit value x1:x0 (two's
// complement) to double: the magnitude's top 64 bits (with a sticky bit for
// the rest) are converted once and scaled by a power of two.
__host__ __device__ __forceinline__ double i128_to_double(unsigned long long x1,
                                                           unsigned long long x0) {
  const bool neg = (long long)x1 < 0;
  if (neg) {  // negate: ~x + 1
    x0 = ~x0 + 1ull;
    x1 = ~x1 + (x0 == 0 ? 1ull : 0ull);
  }
  double mag;
  if (x1 == 0) {
    mag = double(x0);
  } else {
#ifdef __CUDA_ARCH__
    const int lz = __clzll((long long)x1);
#else
    const int lz = __builtin_clzll(x1);
#endif
    const unsigned long long top = lz ? ((x1 << lz) | (x0 >> (64 - lz))) : x1;
    const unsigned long long rest = lz ? (x0 << lz) : x0;
    const double t = double(top | (rest != 0 ? 1ull : 0ull));
#ifdef __CUDA_ARCH__
    mag = t * __longlong_as_double((long long)(1023 + 64 - lz) << 52);  // exact: 2^(64-lz)
#else
    mag = std::ldexp(t, 64 - lz);
#endif
  }
  return neg ? -mag : mag;
}

// X = (sum_t W_t r_t) mod P as a signed value in (-P/2, P/2], converted to double.
// The r_t need not be reduced: any 0 <= r_t < 2^24 congruent to the residue
// works (the INT8 GEMM hands over sums of per-chunk residues).
__host__ __device__ __forceinline__ double crt_value(const int* r, const ReconParams& rp) {
  // S = sum_t W_t r_t accumulated per 32-bit limb of W_t: each product is
  // below 2^56 and at most 16 of them below 2^60, so the four 64-bit limb sums
  // need no carries (one 32x32->64 multiply-add per limb and modulus)
  // (unrolled to the usable maximum so that r stays in registers)
  unsigned long long l0 = 0, l1 = 0, l2 = 0, l3 = 0;
#pragma unroll
  for (int t = 0; t < kMaxUsableModuli; ++t) {
    if (t >= rp.n) break;
    const unsigned long long rt = (unsigned int)r[t];
    l0 += rt * (unsigned int)rp.w_lo[t];
    l1 += rt * (unsigned int)(rp.w_lo[t] >> 32);
    l2 += rt * (unsigned int)rp.w_hi[t];
    l3 += rt * (unsigned int)(rp.w_hi[t] >> 32);
  }
  // carry-propagate into the 192-bit S = s2:s1:s0
  unsigned long long c = l0;
  const unsigned long long d0 = c & 0xFFFFFFFFull;
  c = (c >> 32) + l1;
  const unsigned long long d1 = c & 0xFFFFFFFFull;
  c = (c >> 32) + l2;
  const unsigned long long d2 = c & 0xFFFFFFFFull;
  c = (c >> 32) + l3;
  const unsigned long long d3 = c & 0xFFFFFFFFull;
  const unsigned long long s0 = d0 | (d1 << 32), s1 = d2 | (d3 << 32), s2 = c >> 32;
  // q = floor(S / P) estimated in double, then S - qP. S / P < 16 * 2^24 and
  // the estimate S_d * (1 / P_d) carries at most ~6 roundings of 2^-53
  // relative, an absolute error below 2^-22: q is off by at most one, and one
  // conditional add or subtract of P brings S - qP into [0, P).
  const double S_d = double(s2) * 3.402823669209385e38 + double(s1) * 18446744073709551616.0 +
                     double(s0);
  unsigned long long q = (unsigned long long)floor(S_d * rp.inv_P);
  // qP (192-bit)
  const unsigned long long qp0 = rp.P_lo * q, qp0h = mulhi64(rp.P_lo, q);
  const unsigned long long qp1l = rp.P_hi * q, qp1h = mulhi64(rp.P_hi, q);
  unsigned long long t1 = qp0h + qp1l;
  unsigned long long t2 = qp1h + (t1 < qp0h);
  // X = S - qP (192-bit two's complement)
  unsigned long long x0 = s0 - qp0;
  unsigned long long br = s0 < qp0;
  unsigned long long x1 = s1 - t1 - br;
  unsigned long long br1 = (s1 < t1) || (s1 - t1 < br);
  unsigned long long x2 = s2 - t2 - br1;
  // fix-up into [0, P)
  {
    if ((long long)x2 < 0) {  // X < 0: X += P
      unsigned long long n0 = x0 + rp.P_lo;
      unsigned long long cy = n0 < x0;
      unsigned long long n1 = x1 + rp.P_hi + cy;
      unsigned long long cy1 = (n1 < x1) || (cy && n1 == x1);
      x0 = n0;
      x1 = n1;
      x2 += cy1;
    } else if (x2 > 0 || x1 > rp.P_hi || (x1 == rp.P_hi && x0 >= rp.P_lo)) {  // X >= P
      unsigned long long n0 = x0 - rp.P_lo;
      unsigned long long b0 = x0 < rp.P_lo;
      unsigned long long n1 = x1 - rp.P_hi - b0;
      unsigned long long b1 = (x1 < rp.P_hi) || (x1 - rp.P_hi < b0);
      x0 = n0;
      x1 = n1;
      x2 -= b1;
    }
  }
  // now 0 <= X < P (x2 == 0). Symmetric: X > P/2 -> X - P.
  const unsigned long long hP_hi = rp.P_hi >> 1,
                           hP_lo = (rp.P_lo >> 1) | (rp.P_hi << 63);
  const bool upper = x1 > hP_hi || (x1 == hP_hi && x0 > hP_lo);
  if (upper) {
    const unsigned long long n0 = x0 - rp.P_lo;
    const unsigned long long b0 = x0 < rp.P_lo;
    const unsigned long long n1 = x1 - rp.P_hi - b0;
    x0 = n0;
    x1 = n1;  // now the top limb is negative (two's complement 128-bit)
  }
  return i128_to_double(x1, x0);
}


}  // namespace oz
}  // namespace splab
