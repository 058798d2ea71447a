// Ozaki scheme II contraction on INT8 tensor cores (tcgen05, sm_100a).
//
// C <- alpha * op(A) * op(B) + beta * C for float / double / complex with
// op(A), op(B) in {N, T, C} (the layouts of pgemm_ssb, K-major operands,
// reference src/pgemm_ssb/pgemm_ssb_host.cpp:168-171, of pgemm_sbs and of
// gemm; op(A) = N and op(B) = T, C are read in place, see 2a).
//
// Method (Ozaki, Uchino & Imamura, "Ozaki Scheme II: A GEMM-oriented emulation
// of floating-point matrix multiplication using an integer modular
// technique", 2025), restated here in our own formulation:
//   1. Complex products as three real ones (Karatsuba): with a = ar + i ai
//      and b = br + i bi, P0 = ar.br, P1 = ai.bi, P2 = (ar + s ai).(br + bi),
//      s = -1 for A^H (Re = P0 + P1, Im = P2 - P0 + P1) and +1 otherwise
//      (Re = P0 - P1, Im = P2 - P0 - P1). Each is a real GEMM of depth k;
//      the combination happens on the residues, before the reconstruction.
//   2. Scaling. Every row x (complex: its interleaved reals) is scaled by
//      2^sigma so that ||2^sigma x||_2 < 2^Q and rounded to integers A', B'
//      (exact in double). By Cauchy-Schwarz every entry of the real product,
//      and Re and Im of the complex one, is below 2^(2Q) <= P/4.
//   3. Residues. For pairwise coprime moduli p_t <= 256 with product P, the
//      residues of A', B' mod p_t (symmetric, int8; the third complex plane
//      is the reduced sum of the first two) are multiplied exactly on the
//      INT8 tensor cores with INT32 accumulation (k-chunks of at most 124928
//      so that 128*128*chunk < 2^31), reduced mod p_t and summed over chunks.
//   4. Reconstruction. The Chinese remainder theorem gives X exactly (|X| <=
//      P/4, so the quotient S/P rounds to the right integer without
//      correction); C = 2^(-sigma_i - tau_j) X, then alpha/beta.
// The only rounding is the integer rounding of step 2 (relative to each row's
// 2-norm, 2^-Q) and the final conversion of X to double.
//
// Kernels: oz_row_scale (row norms -> sigma), oz_slice (scaled residues,
// int8, K-major, one plane per modulus and product), oz_row_scale_mn /
// oz_slice_mn (the same for op(A) = N and op(B) = T, C read in place),
// oz_transpose (op(A) = N copied K-major when k is too long for that),
// oz_slice_tc (opt-in: digit sums on the tensor cores), oz_gemm_pair / oz_gemm
// (tcgen05.mma kind::i8, TMA-fed, TMEM accumulators, warp-specialised
// persistent kernels), oz_reconstruct_tc (CRT sums on the tensor cores) and
// oz_reconstruct / oz_reconstruct_staged (CRT on the CUDA cores), each with
// scaling, alpha/beta and fill-mode tile skipping into C.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "ozaki.cuh"
#include "ozaki_crt.cuh"
#include "tcgen05_common.cuh"

namespace splab {
namespace oz {
using namespace tc;

constexpr int BM = 128;       // rows of A per tile (TMEM lanes)
constexpr int BN = 256;       // rows of B per tile (TMEM columns)
constexpr int BKB = 128;      // k bytes per pipeline stage (one 128-byte swizzle atom)
constexpr int STAGES = 4;
constexpr int A_STAGE = BM * BKB;  // 16 KiB
constexpr int B_STAGE = BN * BKB;  // 32 KiB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int GEMM_THREADS = 192;  // warp 0: TMA, warp 1: MMA, warps 2-5: epilogue
constexpr int GEMM_SMEM = STAGES * STAGE_BYTES + 1024 /*barriers*/ + 1024 /*alignment*/;
// Max k (bytes) per INT32 accumulation: 127/128 * 128 * 128 * chunk < 2^31.
constexpr int kChunkBlocks = 976;  // 976 * 128 = 124928
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s bound on any wait

// --------------------------------------------------------------------------
// device helpers

// Instruction descriptor of tcgen05.mma kind::i8: S32 accumulate, signed int8
// A and B, both K-major, M = 128, N = 256.
constexpr uint32_t kIdescI8 = (2u << 4)              // D format S32
                              | (1u << 7)            // A format: signed int8
                              | (1u << 10)           // B format: signed int8
                              | (uint32_t(BN >> 3) << 17)  // N / 8
                              | (uint32_t(BM >> 4) << 24); // M / 16

// the same with an explicit instruction descriptor
__device__ __forceinline__ void umma_i8_desc(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t accumulate) {
  umma_i8_desc(tmem_d, adesc, bdesc, kIdescI8, accumulate);
}


// --------------------------------------------------------------------------
// 1. row scale exponents

// One block per row: sigma = Q - e where ||row||_2 = f 2^e, f in [0.5, 1).
// Rows of zeros get sigma = 0, rows holding a NaN or an infinity get
// kSigmaNonFinite (the reconstruction then writes NaN where they contribute).
// The sum of squares is kept as S 2^(2E) with E the largest exponent seen
// (rescaled by exact powers of two when it grows), so rows of any finite
// magnitude, 1e-300 or 1e300, neither underflow nor overflow.
constexpr int kSigmaNonFinite = -(1 << 30);

// frexp-style exponent of |v| (v = f 2^e, f in [0.5, 1)); subnormals and
// zero as -1022, infinities and NaN as 1025
__device__ __forceinline__ int exponent_of(double v) {
  const int b = int((__double_as_longlong(v) >> 52) & 0x7FF);
  return (b == 0 ? 1 : b) - 1022;
}

__device__ __forceinline__ void scaled_add(double& S, int& E, double S2, int E2) {
  if (E2 > E) {
    S = ldexp(S, 2 * (E - E2)) + S2;
    E = E2;
  } else {
    S += ldexp(S2, 2 * (E2 - E));
  }
}

// Sum of squares of x[0 .. len), thread t taking t, t + blockDim.x, ...,
// into (S, E, inv): batches of 8 independent loads (memory-level
// parallelism), one exponent check per batch.
template <typename TIn>
__device__ __forceinline__ void ssq_row(const TIn* __restrict__ x, int64_t len, double& S, int& E,
                                        double& inv) {
  const int64_t step = blockDim.x;
  int64_t l = threadIdx.x;
  for (; l + 7 * step < len; l += 8 * step) {
    double v[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) v[b] = double(x[l + b * step]);
    int em = exponent_of(v[0]);
#pragma unroll
    for (int b = 1; b < 8; ++b) em = max(em, exponent_of(v[b]));
    if (em > E) {  // rare: rescale the sum to the new largest exponent
      S = ldexp(S, 2 * (E - em));
      E = em;
      inv = ldexp(1.0, -E);
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const double w = v[b] * inv;
      S = fma(w, w, S);
    }
  }
  for (; l < len; l += step) {
    const double v = double(x[l]);
    const int ev = exponent_of(v);
    if (ev > E) {
      S = ldexp(S, 2 * (E - ev));
      E = ev;
      inv = ldexp(1.0, -E);
    }
    const double w = v * inv;
    S = fma(w, w, S);
  }
}

// Sum of squares of a sample of a row: nruns runs of run reals, gap apart;
// blockDim.x / nruns threads per run (blockDim.x a multiple of nruns),
// batches of 8 independent loads along it (the runs are short).
template <typename TIn>
__device__ __forceinline__ void ssq_sample(const TIn* __restrict__ x, int nruns, int64_t run,
                                           int64_t gap, double& S, int& E, double& inv) {
  const int gsz = int(blockDim.x) / nruns;
  const int c = int(threadIdx.x) / gsz;
  if (c >= nruns) return;
  x += c * gap;
  for (int64_t l = threadIdx.x % gsz; l < run; l += 8 * gsz) {
    double v[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) v[b] = l + b * gsz < run ? double(x[l + b * gsz]) : 0.0;
    int em = exponent_of(v[0]);
#pragma unroll
    for (int b = 1; b < 8; ++b) em = max(em, exponent_of(v[b]));
    if (em > E) {
      S = ldexp(S, 2 * (E - em));
      E = em;
      inv = ldexp(1.0, -E);
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const double w = v[b] * inv;
      S = fma(w, w, S);
    }
  }
}

// The block's (S, E) summed into thread 0's (blocks of at most 1024 threads)
__device__ __forceinline__ void block_ssq(double& S, int& E, double* redS, int* redE) {
  for (int o = 16; o > 0; o >>= 1) {
    const double S2 = __shfl_xor_sync(0xffffffffu, S, o);
    const int E2 = __shfl_xor_sync(0xffffffffu, E, o);
    scaled_add(S, E, S2, E2);
  }
  if ((threadIdx.x & 31) == 0) {
    redS[threadIdx.x >> 5] = S;
    redE[threadIdx.x >> 5] = E;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool have = threadIdx.x < (blockDim.x >> 5);
    S = have ? redS[threadIdx.x] : 0.0;
    E = have ? redE[threadIdx.x] : -2100;
    for (int o = 16; o > 0; o >>= 1) {
      const double S2 = __shfl_xor_sync(0xffffffffu, S, o);
      const int E2 = __shfl_xor_sync(0xffffffffu, E, o);
      scaled_add(S, E, S2, E2);
    }
  }
}

// Estimated norms whose mantissa (in [0.5, 1)) lies within this relative
// distance of either end of its octave take the exact norm instead.
constexpr double kEstimateBand = 1.0 / 32;

// One block per row (with a list, the blocks walk the rows list[0 .. *count
// - 1], grid-stride; else block b takes row b); len reals per row.
// With nruns > 0 the row's exponent is first estimated from a sample (nruns
// runs of run reals, gap apart; the sum of squares extrapolated to len
// reals) and kept when its norm's mantissa is clear of the octave's ends by
// kEstimateBand (exact[row] = 0); otherwise, and for a zero or non-finite
// sample, the whole row is read (exact[row] = 1) as without a sample.
template <typename TIn>
__global__ void oz_row_scale(const TIn* __restrict__ X, int64_t ld_elems, int64_t len, int rows,
                             int q_bits, int* __restrict__ sigma,
                             const int* __restrict__ list = nullptr,
                             const int* __restrict__ count = nullptr, int nruns = 0,
                             int64_t run = 0, int64_t gap = 0, int* __restrict__ exact = nullptr) {
  __shared__ double redS[32];
  __shared__ int redE[32];
  __shared__ int use_estimate;
  const int nwork = list ? *count : min(rows, int(gridDim.x));
  for (int bi = blockIdx.x; bi < nwork; bi += gridDim.x) {
    const int row = list ? list[bi] : bi;
    const TIn* x = X + int64_t(row) * ld_elems;
    double S = 0.0, inv = 0.0;  // sum of (v 2^-E)^2, and 2^-E
    int E = -2100;              // below any exponent: the first batch sets it
    if (nruns > 0) {
      ssq_sample(x, nruns, run, gap, S, E, inv);
      block_ssq(S, E, redS, redE);
      if (threadIdx.x == 0) {
        bool use = false;
        if (S > 0.0 && S < 1e300) {
          int e0 = 0;
          const double f = frexp(sqrt(S * (double(len) / double(nruns * run))), &e0);
          use = f > 0.5 * (1.0 + kEstimateBand) && f < 1.0 - kEstimateBand;
          if (use) sigma[row] = q_bits - (e0 + E);
        }
        exact[row] = use ? 0 : 1;
        use_estimate = use;
      }
      __syncthreads();
      const bool done = use_estimate;
      S = 0.0;
      inv = 0.0;
      E = -2100;
      if (done) continue;  // block-uniform; the next row's first barrier
                           // comes after this row's last read of use_estimate
    }
    ssq_row(x, len, S, E, inv);
    block_ssq(S, E, redS, redE);
    if (threadIdx.x == 0) {
      if (!(S < 1e300)) {  // NaN or infinite input
        sigma[row] = kSigmaNonFinite;
      } else if (S > 0.0) {
        int e0 = 0;
        frexp(sqrt(S), &e0);
        sigma[row] = q_bits - (e0 + E);
      } else {
        sigma[row] = 0;
      }
    }
    __syncthreads();  // redS / redE are reused by the block's next row
  }
}

// --------------------------------------------------------------------------
// 2. residues

// Per-modulus constants of the slicer, each stored twice (both halves of an
// f32x2 operand): -p, 1/p and the digit weights b^i mod p in symmetric form,
// i = 1..4 (digit base b = 2^15 with four digits, else 2^13).
struct SliceConsts {
  int n;
  float p0;  // first modulus (256: residue = low byte of the lowest digit)
  unsigned long long neg_p[kMaxModuli];
  unsigned long long inv_p[kMaxModuli];
  unsigned long long c[kMaxModuli][4];
};

// Residues are computed on the FP32 pipe from digits of the scaled integer
// x = round(2^sigma y), x = sum_i d_i b^i, which are extracted without
// conversion instructions: x = xh 2^h + xl with xh = round(y 2^-h), both read
// as integers from the bits of (value + 1.5 2^52).
//   NDIG 3 and 5 (|x| < 2^39, < 2^62): b = 2^13, h = 26; d_0 = xl mod 2^13
//     (0 .. 8191), d_1 = xl >> 13 (|d_1| <= 4096), xh gives d_2.. the same
//     way (top digit signed); the digit sum below stays under 2^22.
//   NDIG 4 (|x| < 2^58, the default for double): b = 2^15, h = 30, balanced
//     digits (|d_0|, |d_1|, |d_2| <= 2^14 + 1, |d_3| <= 2^13 + 1): one digit
//     fewer; the digit sum stays under 5.3e6 < 2^23.
// For a modulus p the digit sum s = d_0 + sum_i c_i d_i (c_i = b^i mod p in
// symmetric form, |c_i| <= p/2) is exact in FP32, and since |s| < 2^23 the
// quotient rounded from s * fl(1/p) is the nearest integer to s / p (for odd
// p, s / p is at least 1/(2p) away from a half-integer; the product's error is
// below that); r = s - p * nearest(s / p) lies in [-(p-1)/2, (p-1)/2]. For
// p = 256 the weights vanish and r is the low byte of d_0. Each residue is
// produced as the float MAGIC + r, whose low byte is r in two's complement:
// the int8 value without a conversion.
__device__ __forceinline__ float small_int_to_float(int d) {  // |d| < 2^22
  return __int_as_float(0x4B400000 + d) - 12582912.0f;
}

template <int NDIG>
__device__ __forceinline__ void digits13(double y, float (&d)[5]) {
  constexpr double kM52 = 6755399441055744.0;  // 1.5 * 2^52: ulp 1
  constexpr long long kM52Bits = 0x4338000000000000ll;
  if (NDIG == 4) {  // balanced base-2^15 digits, |x| < 2^58
    const double t = fma(y, 1.0 / 1073741824.0, kM52);  // kM52 + round(y 2^-30)
    const double xl_d = fma(t - kM52, -1073741824.0, y);  // exact, |xl_d| <= 2^29
    const int xl = int(__double2loint(xl_d + kM52));
    const int xh = int(__double_as_longlong(t) - kM52Bits);  // |xh| <= 2^28 + 1
    // balanced digits: with u = x + 2^14, d_lo = (u mod 2^15) - 2^14 and
    // d_hi = (x - d_lo) / 2^15 = floor(u / 2^15)
    const int u0 = xl + 0x4000, u2 = xh + 0x4000;
    d[0] = small_int_to_float((u0 & 0x7FFF) - 0x4000);
    d[1] = small_int_to_float(u0 >> 15);
    d[2] = small_int_to_float((u2 & 0x7FFF) - 0x4000);
    d[3] = small_int_to_float(u2 >> 15);
    d[4] = 0.0f;
    return;
  }
  const double t = fma(y, 1.0 / 67108864.0, kM52);  // kM52 + round(y 2^-26)
  const double xl_d = fma(t - kM52, -67108864.0, y);  // exact, |xl_d| <= 2^25
  const int xl = int(__double2loint(xl_d + kM52));  // round(xl_d), two's complement
  const long long xh = __double_as_longlong(t) - kM52Bits;
  d[0] = small_int_to_float(xl & 0x1FFF);
  d[1] = small_int_to_float(xl >> 13);
  if (NDIG == 3) {
    d[2] = small_int_to_float(int(xh));
  } else {
    d[2] = small_int_to_float(int(xh & 0x1FFF));
    d[3] = small_int_to_float(int((xh >> 13) & 0x1FFF));
    d[4] = small_int_to_float(int(xh >> 26));
  }
#pragma unroll
  for (int i = NDIG; i < 5; ++i) d[i] = 0.0f;
}

constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: ulp 1, low mantissa bits hold r

// Two floats in one 64-bit register for the packed FP32 instructions of
// sm_100 (fma/add .f32x2: one instruction, two lanes of work).
__host__ __device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
#ifdef __CUDA_ARCH__
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
#else
  uint32_t a, b;
  std::memcpy(&a, &lo, 4);
  std::memcpy(&b, &hi, 4);
  return (static_cast<unsigned long long>(b) << 32) | a;
#endif
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

__device__ __forceinline__ uint32_t pack4(float a, float b, float c, float d) {
  const uint32_t t0 = __byte_perm(__float_as_uint(a), __float_as_uint(b), 0x0040);
  const uint32_t t1 = __byte_perm(__float_as_uint(c), __float_as_uint(d), 0x0040);
  return __byte_perm(t0, t1, 0x5410);
}


// The work of one slicing thread once its EL reals (of one row, starting at
// real l0) are loaded: scaling by 2^sg, digits, and for every modulus the
// residues written to res_row + l0 (mode 0) or, in mode 2, to the three
// planes `plane` bytes apart at complex offset l0 / 2. SSQ: the sum of
// squares of the scaled values is handed to on_ssq once the digits are made
// (so that it is not kept in registers through the residue loop).
struct NoSsq {
  __device__ void operator()(double) const {}
};
template <typename TIn, int NDIG, int EL, int NMU, int MODE, bool SSQ = false,
          typename OnSsq = NoSsq>
__device__ __forceinline__ void slice_thread(double (&v)[EL], int sg, int8_t* res_row,
                                             int64_t l0, int64_t plane, int s_sum,
                                             int64_t res_mod_stride, const SliceConsts& sc,
                                             int t_begin, int t_end, OnSsq on_ssq = {}) {
  static_assert(EL == 8 || EL == 16, "8 or 16 reals per thread");
  static_assert(MODE == 0 || MODE == 2, "real rows or complex rows");
  constexpr int W = EL / 4;  // packed words per modulus
  // 2^sg as a double when representable, else ldexp per element
  const bool direct = sg > -1000 && sg < 1000;
  const double scale = direct ? __longlong_as_double((long long)(sg + 1023) << 52) : 1.0;
  unsigned long long dp[EL / 2][5];  // digits of the element pairs (see below)
  double ssq = 0.0;
  {
    // pairs (2i, 2i + 1) in mode 0; in mode 2 the real parts pair up first,
    // then the imaginary parts: (re0, re1), (re2, re3), ..., (im0, im1), ...
    if constexpr (MODE == 2) {
      double u[EL];
#pragma unroll
      for (int i = 0; i < EL / 2; ++i) {
        u[i] = v[2 * i];
        u[EL / 2 + i] = v[2 * i + 1];
      }
#pragma unroll
      for (int i = 0; i < EL; ++i) v[i] = u[i];
    }
#pragma unroll
    for (int i = 0; i < EL / 2; ++i) {
      float d0[5], d1[5];
      const double y0 = direct ? v[2 * i] * scale : ldexp(v[2 * i], sg);
      const double y1 = direct ? v[2 * i + 1] * scale : ldexp(v[2 * i + 1], sg);
      if constexpr (SSQ) ssq = fma(y1, y1, fma(y0, y0, ssq));
      digits13<NDIG>(y0, d0);
      digits13<NDIG>(y1, d1);
#pragma unroll
      for (int j = 0; j < 5; ++j) dp[i][j] = f2_pack(d0[j], d1[j]);
    }
    if constexpr (SSQ) on_ssq(ssq);
  }
  const unsigned long long M2 = f2_pack(kMagic, kMagic), NM2 = f2_pack(-kMagic, -kMagic);
  int8_t* const out0 = res_row + l0;
  auto modulus = [&](const int t) {
    int8_t* out = out0 + t * res_mod_stride;
    constexpr int H = EL / 4;        // mode 2: pairs of complex elements
    unsigned long long rp2[EL / 2];  // MAGIC + residue of elements 2i, 2i + 1
    unsigned long long ri2[H];       // mode 2: residues of the imaginary pairs, unbiased
    if (t == 0 && sc.p0 == 256.0f) {
#pragma unroll
      for (int i = 0; i < EL / 2; ++i) rp2[i] = f2_add(dp[i][0], M2);
      if constexpr (MODE == 2) {
#pragma unroll
        for (int h = 0; h < H; ++h) ri2[h] = dp[H + h][0];
      }
    } else {
      const unsigned long long np = sc.neg_p[t], ip = sc.inv_p[t];
      const unsigned long long c1 = sc.c[t][0], c2 = sc.c[t][1], c3 = sc.c[t][2],
                               c4 = sc.c[t][3];
#pragma unroll
      for (int i = 0; i < EL / 2; ++i) {
        unsigned long long s2 = f2_fma(c1, dp[i][1], dp[i][0]);
        if (NDIG > 2) s2 = f2_fma(c2, dp[i][2], s2);
        if (NDIG > 3) s2 = f2_fma(c3, dp[i][3], s2);
        if (NDIG > 4) s2 = f2_fma(c4, dp[i][4], s2);
        const unsigned long long q2 = f2_add(f2_fma(s2, ip, M2), NM2);
        // |s| may exceed 2^22 with four digits (s + MAGIC is not exact): r
        // first, then MAGIC + r; both exact. Otherwise one operation fewer.
        if (NDIG == 4 || (MODE == 2 && i >= H)) {
          const unsigned long long r2 = f2_fma(q2, np, s2);
          rp2[i] = f2_add(r2, M2);
          if (MODE == 2 && i >= H) ri2[i - H] = r2;
        } else {
          rp2[i] = f2_fma(q2, np, f2_add(s2, M2));
        }
      }
    }
    float r[EL];
#pragma unroll
    for (int i = 0; i < EL / 2; ++i) f2_unpack(rp2[i], r[2 * i], r[2 * i + 1]);
    uint32_t wu[W];
    if constexpr (MODE == 0) {
#pragma unroll
      for (int q = 0; q < W; ++q)
        wu[q] = pack4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
      if constexpr (W == 4)
        *reinterpret_cast<uint4*>(out) = make_uint4(wu[0], wu[1], wu[2], wu[3]);
      else
        *reinterpret_cast<uint2*>(out) = make_uint2(wu[0], wu[1]);
    } else {
      // rp2[h] = MAGIC + residues of (re_2h, re_2h+1), rp2[H + h] those of the
      // imaginary parts (ri2[h] without MAGIC). Third plane: t = r(re) +
      // s_sum r(im) (|t| < 2^16): MAGIC + t exactly in one FMA, t, its nearest
      // quotient by p and MAGIC + (t - q p) = (MAGIC + t) - q p (for p = 256
      // the residues are unreduced low bytes and the reduction gives the low
      // byte of the sum)
      const unsigned long long np = sc.neg_p[t], ip = sc.inv_p[t];
      const unsigned long long S2 = f2_pack(float(s_sum), float(s_sum));
      unsigned long long sm2[H];
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const unsigned long long tM = f2_fma(S2, ri2[h], rp2[h]);
        const unsigned long long t2 = f2_add(tM, NM2);
        const unsigned long long q2 = f2_add(f2_fma(t2, ip, M2), NM2);
        sm2[h] = f2_fma(q2, np, tM);
      }
      int8_t* o = out0 - l0 + l0 / 2 + t * res_mod_stride;  // complex offset l0 / 2
#pragma unroll
      for (int w = 0; w < H / 2; ++w) {
        float a0, a1, a2, a3;
        f2_unpack(rp2[2 * w], a0, a1);
        f2_unpack(rp2[2 * w + 1], a2, a3);
        *reinterpret_cast<uint32_t*>(o + 4 * w) = pack4(a0, a1, a2, a3);
        f2_unpack(rp2[H + 2 * w], a0, a1);
        f2_unpack(rp2[H + 2 * w + 1], a2, a3);
        *reinterpret_cast<uint32_t*>(o + plane + 4 * w) = pack4(a0, a1, a2, a3);
        f2_unpack(sm2[2 * w], a0, a1);
        f2_unpack(sm2[2 * w + 1], a2, a3);
        *reinterpret_cast<uint32_t*>(o + 2 * plane + 4 * w) = pack4(a0, a1, a2, a3);
      }
    }
  };
  if constexpr (NMU > 0) {
#pragma unroll
    for (int t = 0; t < NMU; ++t) modulus(t);
  } else {
    for (int t = t_begin; t < t_end; ++t) modulus(t);
  }
}

// Residues of one operand, written K-major (row stride kp bytes).
// Each thread handles EL (8 or 16) consecutive reals of one row.
// mode 0: real rows: res[t][row][l], l < kp.
// mode 2: complex rows for the three-product (Karatsuba) form: complex element
//         e = (re, im) of row `row` goes to three planes of `rows` x kp bytes,
//         res[t][0][row][e] = r(re), res[t][1][row][e] = r(im) and
//         res[t][2][row][e] = r(re + s_sum im) (residues are linear in the
//         scaled integers, so the third is r(re) + s_sum r(im) reduced mod p).
//         The input row then holds 2 kp reals (kp complex elements).
// TIn: double (|x| < 2^62, five digits) or float (|x| < 2^38, three digits).
// NMU > 0: moduli 0 .. NMU-1 in one fully unrolled pass (the per-modulus
// constants become fixed parameter operands); 0: t_begin .. t_end-1 in a loop.
// MODE (0 or 2, the mode above) is a template parameter so that the unrolled
// modulus loop carries no branch on it.
// The EL reals of one row at real l0 (zeros past len); VEC: 16-byte loads.
template <typename TIn, bool VEC, int EL>
__device__ __forceinline__ void load_reals(const TIn* __restrict__ x, int64_t l0, int64_t len,
                                           double (&v)[EL]) {
  if (VEC && l0 + EL <= len) {
    if constexpr (sizeof(TIn) == 8) {
#pragma unroll
      for (int i = 0; i < EL / 2; ++i) {
        const double2 t = __ldg(reinterpret_cast<const double2*>(x) + i);
        v[2 * i] = t.x;
        v[2 * i + 1] = t.y;
      }
    } else {
#pragma unroll
      for (int i = 0; i < EL / 4; ++i) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(x) + i);
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < EL; ++i) v[i] = (l0 + i < len) ? double(x[i]) : 0.0;
  }
}

// SSQ: also adds each row's sum of squares of the scaled values to
// rowssq[row] (one atomic per row and block; blocks of 256 threads).
template <typename TIn, bool VEC, int NDIG, int EL, int NMU, int MODE, bool SSQ = false>
__global__ void __launch_bounds__(256, EL == 8 ? 4 : 2)
    oz_slice(const TIn* __restrict__ X, int64_t ld_doubles, int64_t len, int rows, int64_t kp,
             const int* __restrict__ sigma, int s_sum, int8_t* __restrict__ res,
             int64_t res_mod_stride, SliceConsts sc, int t_begin, int t_end,
             double* __restrict__ rowssq) {
  const int64_t groups = (MODE == 2 ? 2 * kp : kp) / EL;
  const int64_t gid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if constexpr (!SSQ) {
    const int row = int(gid / groups);
    if (row >= rows) return;
    const int64_t l0 = (gid % groups) * EL;
    double v[EL];
    load_reals<TIn, VEC, EL>(X + int64_t(row) * ld_doubles + l0, l0, len, v);
    slice_thread<TIn, NDIG, EL, NMU, MODE>(v, sigma[row], res + int64_t(row) * kp, l0,
                                           int64_t(rows) * kp, s_sum, res_mod_stride, sc, t_begin,
                                           t_end);
  } else {
    // Threads past the last row redo the last row's last groups (the same
    // bytes to the same places) so that every thread takes part in the
    // reductions; their sums count as zero. Aligned segments of W lanes (W
    // the largest power of two dividing groups, at most 32; at least 8,
    // groups being kp / 8 or kp / 16 with kp a multiple of 128) hold one row
    // each: reduced by shuffles, then the block's segments of one row
    // together, one atomic per row and block (atomics from every warp on the
    // few rows the resident blocks share would serialise).
    __shared__ double seg_sum[32];
    __shared__ int seg_row[32];
    const int W = int(groups & -groups) < 32 ? int(groups & -groups) : 32;
    const int nseg = int(blockDim.x) / W;  // blocks of 256 threads: at most 32
    const int row_in = int(gid / groups);
    const int64_t g_in = gid % groups;
    const bool past = row_in >= rows;
    const int row = past ? rows - 1 : row_in;
    const int64_t l0 = (past ? groups - W + (g_in & (W - 1)) : g_in) * EL;
    double v[EL];
    load_reals<TIn, VEC, EL>(X + int64_t(row) * ld_doubles + l0, l0, len, v);
    auto on_ssq = [&](double ssq) {
      if (past) ssq = 0.0;
      for (int o = 16; o > 0; o >>= 1)
        if (o < W) ssq += __shfl_xor_sync(0xffffffffu, ssq, o);
      if ((threadIdx.x & (W - 1)) == 0) {
        seg_sum[threadIdx.x / W] = ssq;
        seg_row[threadIdx.x / W] = past ? -1 : row;
      }
    };
    slice_thread<TIn, NDIG, EL, NMU, MODE, true>(v, sigma[row], res + int64_t(row) * kp, l0,
                                                 int64_t(rows) * kp, s_sum, res_mod_stride, sc,
                                                 t_begin, t_end, on_ssq);
    __syncthreads();
    if (int(threadIdx.x) < nseg) {
      const int sgi = threadIdx.x, r = seg_row[sgi];
      if (r >= 0 && (sgi == 0 || seg_row[sgi - 1] != r)) {  // first segment of its row
        double t = 0.0;
        for (int u = sgi; u < nseg && seg_row[u] == r; ++u) t += seg_sum[u];
        atomicAdd(rowssq + r, t);
      }
    }
  }
}

// oz_slice over the rows list[0 .. *count - 1] (grid-stride over their
// thread groups): the rows the one-pass check sent back (see oz_onepass_check)
template <typename TIn, bool VEC, int NDIG, int EL, int NMU, int MODE>
__global__ void __launch_bounds__(256, EL == 8 ? 4 : 2)
    oz_slice_rows(const TIn* __restrict__ X, int64_t ld_doubles, int64_t len, int rows,
                  int64_t kp, const int* __restrict__ sigma, int s_sum,
                  int8_t* __restrict__ res, int64_t res_mod_stride, SliceConsts sc,
                  const int* __restrict__ list, const int* __restrict__ count) {
  const int64_t groups = (MODE == 2 ? 2 * kp : kp) / EL;
  const int64_t total = int64_t(*count) * groups;
  for (int64_t gid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; gid < total;
       gid += int64_t(gridDim.x) * blockDim.x) {
    const int row = list[gid / groups];
    const int64_t l0 = (gid % groups) * EL;
    double v[EL];
    load_reals<TIn, VEC, EL>(X + int64_t(row) * ld_doubles + l0, l0, len, v);
    slice_thread<TIn, NDIG, EL, NMU, MODE>(v, sigma[row], res + int64_t(row) * kp, l0,
                                           int64_t(rows) * kp, s_sum, res_mod_stride, sc, 0, NMU);
  }
}

// One-pass row scaling: a row whose exponent was estimated (exact[i] = 0)
// keeps it when its sum of squares at that scale lies within [lo, hi] (the
// exponent is then the exact one, and clear of the rounding of the sum);
// otherwise (the estimate was off, the row is zero or not finite, or the sum
// lies near an exponent boundary) it is listed for its exact norm and a
// second slicing.
__global__ void oz_onepass_check(const double* __restrict__ ssq, const int* __restrict__ exact,
                                 int rows, double lo, double hi, int* __restrict__ list,
                                 int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  const double S = ssq[i];
  if (!exact[i] && !(S >= lo && S <= hi)) list[atomicAdd(count, 1)] = i;
}

// --------------------------------------------------------------------------
// 2a. operands read in place: op(A) = N (A m-major: element (i, kk) at
// X[i + kk ld], the rows of op(A) are the columns of X) and op(B) = T or C
// (B n-major the same way). Instead of a k-major copy the norms read them
// along the rows and the slicer transposes tiles through shared memory.
constexpr int kMnRows = 65536;  // rows from which the norms need no k-slicing

// sigma from the exponent-tracked sum of squares S 2^(2E) of a row
__device__ __forceinline__ int sigma_of(double S, int E, int q_bits) {
  if (!(S < 1e300)) return kSigmaNonFinite;  // NaN or infinite input
  if (S > 0.0) {
    int e0 = 0;
    frexp(sqrt(S), &e0);
    return q_bits - (e0 + E);
  }
  return 0;
}

// Row scale exponents of m-major rows, as oz_row_scale computes them: one
// thread per row and k-slice (a warp reads 32 consecutive rows of one kk:
// coalesced), batches of 8 loads in flight. With one k-slice (gridDim.y == 1)
// the thread writes sigma; with several it writes its partial sum (S, E) to
// partS / partE [slice][row] for oz_row_scale_combine.
template <typename TIn, bool CPLX>
__global__ void __launch_bounds__(256) oz_row_scale_mn(const TIn* __restrict__ X, int64_t ld,
                                                       int m, int64_t k, int64_t kspan, int q_bits,
                                                       int* __restrict__ sigma,
                                                       double* __restrict__ partS,
                                                       int* __restrict__ partE) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  constexpr int R = CPLX ? 2 : 1;  // reals per element
  const TIn* x = X + int64_t(i) * R;
  const int64_t step = ld * R;  // reals between consecutive kk
  double S = 0.0, inv = 0.0;
  int E = -2100;
  int64_t kk = int64_t(blockIdx.y) * kspan;
  const int64_t kend = min(k, kk + kspan);
  for (; kk + 8 <= kend; kk += 8) {
    double v[8 * R];
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int c = 0; c < R; ++c) v[b * R + c] = double(x[(kk + b) * step + c]);
    int em = exponent_of(v[0]);
#pragma unroll
    for (int b = 1; b < 8 * R; ++b) em = max(em, exponent_of(v[b]));
    if (em > E) {
      S = ldexp(S, 2 * (E - em));
      E = em;
      inv = ldexp(1.0, -E);
    }
#pragma unroll
    for (int b = 0; b < 8 * R; ++b) {
      const double w = v[b] * inv;
      S = fma(w, w, S);
    }
  }
  for (; kk < kend; ++kk) {
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const double v = double(x[kk * step + c]);
      const int ev = exponent_of(v);
      if (ev > E) {
        S = ldexp(S, 2 * (E - ev));
        E = ev;
        inv = ldexp(1.0, -E);
      }
      const double w = v * inv;
      S = fma(w, w, S);
    }
  }
  if (gridDim.y == 1) {
    sigma[i] = sigma_of(S, E, q_bits);
  } else {
    partS[int64_t(blockIdx.y) * m + i] = S;
    partE[int64_t(blockIdx.y) * m + i] = E;
  }
}

// sigma of each row from its k-slice partial sums
__global__ void __launch_bounds__(256) oz_row_scale_combine(const double* __restrict__ partS,
                                                            const int* __restrict__ partE, int m,
                                                            int slices, int q_bits,
                                                            int* __restrict__ sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double S = 0.0;
  int E = -2100;
  for (int sl = 0; sl < slices; ++sl)
    scaled_add(S, E, partS[int64_t(sl) * m + i], partE[int64_t(sl) * m + i]);
  sigma[i] = sigma_of(S, E, q_bits);
}

// Raw element of ESZ bytes (a complex or real value of TIn) in shared memory
template <int ESZ> struct RawElem;
template <> struct RawElem<16> { using T = double2; };
template <> struct RawElem<8> { using T = unsigned long long; };
template <> struct RawElem<4> { using T = unsigned int; };

// Residues of m-major rows: a block covers 8 rows (one warp each) and, per row,
// the KT = 32 G elements of one warp row (G = EL / reals per element: 4
// complex or 8 real). The tile is read along i (8 consecutive rows per kk) into
// shared memory and read back along kk; the element index is XOR-swizzled
// within groups of 128 bytes and the row stride is odd, so that the reads are
// free of bank conflicts (the writes at most 2-way, 4-way for real float).
// Each thread then does oz_slice's work (slice_thread) on its EL = 8 reals.
// VEC: 16-byte loads of complex double elements (the base is 16-byte aligned).
// conj: complex elements are conjugated as they are loaded (op(B) = C).
template <typename TIn, bool VEC, int NDIG, int NMU, int MODE>
__global__ void __launch_bounds__(256, 4)
    oz_slice_mn(const TIn* __restrict__ X, int64_t ld, int m, int64_t k, int64_t kp,
                const int* __restrict__ sigma, int s_sum, int conj, int8_t* __restrict__ res,
                int64_t res_mod_stride, SliceConsts sc, int t_begin, int t_end) {
  constexpr int EL = 8;
  constexpr int R = MODE == 2 ? 2 : 1;  // reals per element
  constexpr int G = EL / R;             // elements per thread
  constexpr int KT = 32 * G;            // elements per row per tile
  constexpr int ESZ = R * int(sizeof(TIn));
  constexpr int GROUPS = 128 / ESZ;     // elements per 128 bytes of shared memory
  constexpr int RSTR = KT + 1;          // row stride in elements (odd)
  using T = typename RawElem<ESZ>::T;
  __shared__ T tile[8 * RSTR];
  auto swz = [](int kk) { return kk ^ ((kk / G) & (GROUPS - 1)); };
  const int i0 = blockIdx.x * 8;
  const int64_t kk0 = int64_t(blockIdx.y) * KT;
#pragma unroll
  for (int it = 0; it < KT / 32; ++it) {
    const int r = threadIdx.x & 7, kk = (threadIdx.x >> 3) + 32 * it;
    T val;
    if (i0 + r < m && kk0 + kk < k) {
      const int64_t e = int64_t(i0 + r) + (kk0 + kk) * ld;  // element index
      if constexpr (ESZ == 16) {
        if (VEC) {
          val = __ldg(reinterpret_cast<const double2*>(X) + e);
        } else {
          val.x = double(X[2 * e]);
          val.y = double(X[2 * e + 1]);
        }
      } else if constexpr (ESZ == 8 && sizeof(TIn) == 8) {
        val = __double_as_longlong(double(X[e]));
      } else if constexpr (ESZ == 8) {  // complex float
        val = (static_cast<unsigned long long>(__float_as_uint(float(X[2 * e + 1]))) << 32) |
              __float_as_uint(float(X[2 * e]));
      } else {
        val = __float_as_uint(float(X[e]));
      }
    } else {
      if constexpr (ESZ == 16)
        val = make_double2(0.0, 0.0);
      else
        val = 0;
    }
    tile[r * RSTR + swz(kk)] = val;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int row = i0 + w;
  if (row >= m || kk0 + G * l >= kp) return;
  double v[EL];
#pragma unroll
  for (int q = 0; q < G; ++q) {
    const T e = tile[w * RSTR + swz(G * l + q)];
    if constexpr (ESZ == 16) {
      v[2 * q] = e.x;
      v[2 * q + 1] = conj ? -e.y : e.y;
    } else if constexpr (ESZ == 8 && sizeof(TIn) == 8) {
      v[q] = __longlong_as_double(static_cast<long long>(e));
    } else if constexpr (ESZ == 8) {
      v[2 * q] = double(__uint_as_float(unsigned(e)));
      const double im = double(__uint_as_float(unsigned(e >> 32)));
      v[2 * q + 1] = conj ? -im : im;
    } else {
      v[q] = double(__uint_as_float(e));
    }
  }
  slice_thread<TIn, NDIG, EL, NMU, MODE>(v, sigma[row], res + int64_t(row) * kp,
                                         (kk0 + G * l) * R, int64_t(m) * kp, s_sum,
                                         res_mod_stride, sc, t_begin, t_end);
}

// --------------------------------------------------------------------------
// 2b. residues of complex double rows with the digit sums on the tensor cores
//
// The digit sums above are a small integer matrix product. Written in
// balanced base-256 digits, x = sum_j d_j 256^j with d_j in [-128, 127]
// (eight digits cover |x| < 2^62), the residue of x mod p is that of
// sum_j d_j w_j with w_j = 256^j mod p in symmetric form (|w_j| <= 127). A
// complex element has 16 digits (8 of re, 8 of im), and its three planes are
// three such sums: re uses w on the re digits, im w on the im digits, the
// sum plane w on re and s_sum w on im. One tcgen05.mma kind::i8 (exact INT32)
//   D[128 x 256] = W[128 x K] . Dig[K x 256]
// computes them for G groups of 256 elements at once: the 16 digit bytes of
// group g's element n are K bytes 16 g .. 16 g + 15 of B row n, and row
// (g, t, q) of W holds the weights of modulus t and plane q on group g's
// bytes; (nmod - 1) * 3 * G <= 128 rows (G = 3 for the default 15 moduli:
// 126 rows, two K-steps of 32 bytes). The modulus 256 is the low byte of x and
// is written by the producers directly. The epilogue reduces each sum
// (|s| < 16 * 128 * 127 < 2^18) mod p on the FP32 pipe with 4 operations
// per residue (against 7 for the digit-sum form plus 3 for the sum plane),
// stages the bytes of its 256-element row segment in shared memory and writes
// it with one bulk copy.
//
// Warps 0-7: epilogue (warp w reads TMEM lanes 32 (w % 4) .. + 31, one
// (group, modulus, plane) row each, and columns 128 (w / 4) .. + 127, two
// warps per lane quarter so that the TMEM loads and the reduction of one
// overlap the other's); warps 8-11: producers (row scaling, digits into the
// 128-byte-swizzled B tile, modulus-256 bytes); warp 12: TMEM allocation and
// the MMA issue. Digits and accumulators are double-buffered; every wait is
// bounded and a give-up sets *status. Each epilogue warp stages its 32 row
// segments of 128 bytes in shared memory and writes them with coalesced
// 16-byte stores (4 rows of 128 bytes per instruction; one bulk copy per row
// segment measured 30 % slower: the copy engine's cost per small copy).
struct SliceTcParams {
  const double* X;        // rows of interleaved complex doubles
  int64_t ld;             // row stride in doubles
  int64_t len;            // complex elements per row
  int rows;
  int64_t kp;             // residue row length (complex elements, multiple of 128)
  const int* sigma;       // row scale exponents
  int s_sum;              // sign of im in the third plane
  int8_t* res;            // res[t][q][row][e]
  int64_t mod_stride;     // bytes between moduli
  int64_t plane;          // bytes between the planes of one modulus
  int nmod;               // moduli, p[0] = 256
  int groups;             // groups of 256 elements per unit
  int ksteps;             // K-steps of 32 bytes per unit
  int units_per_row;
  long long total_units;
  int p[kMaxModuli];
  int* status;
  unsigned long long wait_limit_ns;
};

constexpr int TC_THREADS = 416;  // warps 0-7 epilogue, 8-11 producers, 12 MMA
constexpr int TC_W_BYTES = 128 * 128;            // weights: 128 rows x 128 B (SW128)
constexpr int TC_D_BYTES = 256 * 128;            // digits: 256 rows x 128 B (SW128)
constexpr int TC_ROW_STAGE = 256 + 16;           // one staged row segment (padded)
constexpr int TC_S_BYTES = 128 * TC_ROW_STAGE;   // staging of the 128 epilogue rows
constexpr int TC_SMEM = TC_W_BYTES + 2 * TC_D_BYTES + 2 * TC_S_BYTES + 256 + 1024;

__device__ __forceinline__ int sw128_chunk(int row, int chunk) {
  return (row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4);
}

// round(y) as a 64-bit integer for |y| < 2^62, without conversion
// instructions: y = xh 2^30 + xl_d, both parts read from the bits of
// (value + 1.5 2^52).
__device__ __forceinline__ long long round_to_int64(double y) {
  constexpr double kM52 = 6755399441055744.0;  // 1.5 * 2^52: ulp 1
  constexpr long long kM52Bits = 0x4338000000000000ll;
  const double t = fma(y, 1.0 / 1073741824.0, kM52);   // kM52 + round(y 2^-30)
  const double xl_d = fma(t - kM52, -1073741824.0, y);  // exact, |xl_d| <= 2^29
  const long long xh = __double_as_longlong(t) - kM52Bits;
  const int xl = int(__double2loint(xl_d + kM52));
  return xh * 1073741824ll + xl;
}

// Balanced base-256 digits of x as bytes: d_j = byte_j(x + 0x0080..80) - 128
// for j < 7 (the XOR flips the offset back), d_7 the signed top byte.
__device__ __forceinline__ unsigned long long balanced_digits(long long x) {
  constexpr unsigned long long kOff = 0x0080808080808080ull;
  return (static_cast<unsigned long long>(x) + kOff) ^ kOff;
}

__global__ void __launch_bounds__(TC_THREADS, 1) oz_slice_tc(const __grid_constant__ SliceTcParams P) {
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  const uint32_t base = (raw_addr + 1023u) & ~1023u;
  unsigned char* bp = smem_raw + (base - raw_addr);
  unsigned char* Wt = bp;
  unsigned char* Dg = bp + TC_W_BYTES;
  unsigned char* St = Dg + 2 * TC_D_BYTES;
  const uint32_t w_addr = base, d_addr = base + TC_W_BYTES, s_addr = d_addr + 2 * TC_D_BYTES;
  const uint32_t bar_base = s_addr + 2 * TC_S_BYTES;
  auto dfull = [&](int b) { return bar_base + 8u * b; };
  auto dempty = [&](int b) { return bar_base + 8u * (2 + b); };
  auto accf = [&](int b) { return bar_base + 8u * (4 + b); };
  auto acce = [&](int b) { return bar_base + 8u * (6 + b); };
  const uint32_t drain_bar = bar_base + 64;
  unsigned char* tail = St + 2 * TC_S_BYTES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tail + 128);
  volatile int* abort = reinterpret_cast<volatile int*>(tail + 136);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int R3 = 3 * (P.nmod - 1);
  const int wrows = P.groups * R3;

  // weights: row L = (group g, modulus t >= 1, plane q), K byte k
  for (int i = threadIdx.x; i < 128 * 128; i += blockDim.x) {
    const int L = i >> 7, k = i & 127;
    int w = 0;
    if (L < wrows) {
      const int g = L / R3, j = L - g * R3, t = 1 + j / 3, q = j - 3 * (j / 3);
      const int kg = k - 16 * g;
      if (kg >= 0 && kg < 16) {
        const int part = kg >> 3, dj = kg & 7;  // part 0: re digits, 1: im digits
        const int pt = P.p[t];
        int c = 1;
        for (int s = 0; s < dj; ++s) c = (c * 256) % pt;
        if (c > pt / 2) c -= pt;
        if (q == 0) w = part == 0 ? c : 0;
        else if (q == 1) w = part == 1 ? c : 0;
        else w = part == 0 ? c : P.s_sum * c;
      }
    }
    Wt[sw128_chunk(L, k >> 4) + (k & 15)] = static_cast<unsigned char>(static_cast<signed char>(w));
  }
  // digit tiles start at zero: the bytes beyond the groups are read by the
  // last K-step (against zero weights) and never written
  for (int i = threadIdx.x; i < 2 * TC_D_BYTES / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(Dg)[i] = make_uint4(0u, 0u, 0u, 0u);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; ++b) {
      mbar_init(dfull(b), 128);
      mbar_init(dempty(b), 1);
      mbar_init(accf(b), 1);
      mbar_init(acce(b), 256);
    }
    mbar_init(drain_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 12) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     smem_u32(tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int unit_elems = 256 * P.groups;

  if (warp >= 8 && warp < 12) {
    // ---- producers: 2 G elements per thread and unit, consecutive threads
    // on consecutive elements (coalesced 16-byte loads)
    const int pt = threadIdx.x - 256;
    const int per = 2 * P.groups;
    // the elements of unit u, loaded one unit ahead of their use
    auto load = [&](long long u, double2 (&v)[8]) {
      const int row = int(u / P.units_per_row);
      const int64_t e0 = (u - int64_t(row) * P.units_per_row) * unit_elems;
      const double2* xr = reinterpret_cast<const double2*>(P.X + int64_t(row) * P.ld);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        if (r < per) {
          const int64_t e = e0 + pt + 128 * r;
          v[r] = e < P.len ? __ldcs(xr + e) : make_double2(0.0, 0.0);
        }
      }
    };
    double2 v[8], vn[8];
    if (blockIdx.x < P.total_units) load(blockIdx.x, vn);
    for (long long u = blockIdx.x, it = 0; u < P.total_units; u += gridDim.x, ++it) {
      const int b = int(it & 1);
      const uint32_t par = uint32_t((it >> 1) & 1);
      const int row = int(u / P.units_per_row);
      const int64_t e0 = (u - int64_t(row) * P.units_per_row) * unit_elems;
      const int sg = P.sigma[row];
      const bool direct = sg > -1000 && sg < 1000;
      const double scale = direct ? __longlong_as_double((long long)(sg + 1023) << 52) : 1.0;
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = vn[r];
      if (u + gridDim.x < P.total_units) load(u + gridDim.x, vn);
      if (!mbar_wait(dempty(b), par ^ 1u, abort, P.wait_limit_ns)) break;
      unsigned char* dg = Dg + b * TC_D_BYTES;
      int8_t* r256 = P.res + int64_t(row) * P.kp;  // modulus 0 (256), plane 0
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        if (r < per) {
          const int el = pt + 128 * r;
          const int64_t e = e0 + el;
          const double yr = direct ? v[r].x * scale : ldexp(v[r].x, sg);
          const double yi = direct ? v[r].y * scale : ldexp(v[r].y, sg);
          const long long x_re = round_to_int64(yr), x_im = round_to_int64(yi);
          const unsigned long long dr = balanced_digits(x_re), di = balanced_digits(x_im);
          *reinterpret_cast<uint4*>(dg + sw128_chunk(el & 255, el >> 8)) =
              make_uint4(unsigned(dr), unsigned(dr >> 32), unsigned(di), unsigned(di >> 32));
          if (e < P.kp) {
            r256[e] = static_cast<int8_t>(x_re);
            r256[P.plane + e] = static_cast<int8_t>(x_im);
            r256[2 * P.plane + e] = static_cast<int8_t>(x_re + P.s_sum * x_im);
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(dfull(b));
    }
  } else if (warp == 12) {
    if (lane == 0) {
      // ---- MMA issuer
      bool ok = true;
      for (long long u = blockIdx.x, it = 0; u < P.total_units; u += gridDim.x, ++it) {
        const int b = int(it & 1);
        const uint32_t par = uint32_t((it >> 1) & 1);
        if (!mbar_wait(dfull(b), par, abort, P.wait_limit_ns) ||
            !mbar_wait(acce(b), par ^ 1u, abort, P.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + uint32_t(b * 256);
        for (int kk = 0; kk < P.ksteps; ++kk)
          umma_i8(d, umma_desc_sw128(w_addr + kk * 32),
                  umma_desc_sw128(d_addr + b * TC_D_BYTES + kk * 32), kk > 0 ? 1u : 0u);
        umma_commit(dempty(b));
        umma_commit(accf(b));
      }
      if (!ok) {
        umma_commit(drain_bar);  // MMAs may be in flight: wait (bounded) until they retire
        const unsigned long long t0 = globaltimer();
        while (!mbar_try_wait(drain_bar, 0) && globaltimer() - t0 < 1000000ull) {
        }
      }
    }
  } else if (warp < 8) {
    // ---- epilogue: TMEM lane L = (group, modulus, plane) row, half of the columns
    const int quarter = warp & 3, half = warp >> 2;
    const int L = quarter * 32 + lane;
    const bool active = L < wrows;
    int g = 0, t = 1, q = 0;
    if (active) {
      g = L / R3;
      const int j = L - g * R3;
      t = 1 + j / 3;
      q = j - 3 * (j / 3);
    }
    const float pf = float(P.p[t]);
    const unsigned long long NP2 = f2_pack(-pf, -pf);
    const unsigned long long IP2 = f2_pack(1.0f / pf, 1.0f / pf);
    const unsigned long long M2 = f2_pack(kMagic, kMagic), NM2 = f2_pack(-kMagic, -kMagic);
    const uint32_t seg_stage = uint32_t(L) * TC_ROW_STAGE + uint32_t(half * 128);
    const uint32_t lane_taddr = tmem_base + (uint32_t(quarter * 32) << 16) + uint32_t(half * 128);
    // 32 sums -> 32 residue bytes at st
    auto reduce32 = [&](const uint32_t (&v)[32], unsigned char* st) {
      uint32_t wv[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        float r[4];
#pragma unroll
        for (int e2 = 0; e2 < 2; ++e2) {
          const int c = 4 * h + 2 * e2;
          // MAGIC + s exactly (|s| < 2^22), s, its nearest quotient by p,
          // MAGIC + s - q p = MAGIC + (s mod p)
          const unsigned long long tM = f2_pack(__int_as_float(0x4B400000 + int(v[c])),
                                                __int_as_float(0x4B400000 + int(v[c + 1])));
          const unsigned long long t2 = f2_add(tM, NM2);
          const unsigned long long q2 = f2_add(f2_fma(t2, IP2, M2), NM2);
          f2_unpack(f2_fma(q2, NP2, tM), r[2 * e2], r[2 * e2 + 1]);
        }
        wv[h] = pack4(r[0], r[1], r[2], r[3]);
      }
      *reinterpret_cast<uint4*>(st) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
      *reinterpret_cast<uint4*>(st + 16) = make_uint4(wv[4], wv[5], wv[6], wv[7]);
    };
    for (long long u = blockIdx.x, it = 0; u < P.total_units; u += gridDim.x, ++it) {
      const int b = int(it & 1);
      const uint32_t par = uint32_t((it >> 1) & 1);
      if (!mbar_wait(accf(b), par, abort, P.wait_limit_ns)) break;
      tc_fence_after();
      unsigned char* st = St + b * TC_S_BYTES + seg_stage;
      const uint32_t taddr = lane_taddr + uint32_t(b * 256);
      // four chunks of 32 columns; the load of chunk c + 1 is in flight while
      // chunk c is reduced
      uint32_t va[32], vb[32];
      tmem_ld32_nowait(taddr, va);
      tmem_wait_ld();
      tmem_ld32_nowait(taddr + 32, vb);
      if (active) reduce32(va, st);
      tmem_wait_ld();
      tmem_ld32_nowait(taddr + 64, va);
      if (active) reduce32(vb, st + 32);
      tmem_wait_ld();
      tmem_ld32_nowait(taddr + 96, vb);
      if (active) reduce32(va, st + 64);
      tmem_wait_ld();
      tc_fence_before();
      mbar_arrive(acce(b));  // TMEM buffer b is free for the MMA of unit it + 2
      if (active) reduce32(vb, st + 96);
      const int row = int(u / P.units_per_row);
      const int64_t e_unit = (u - int64_t(row) * P.units_per_row) * unit_elems;
      // this lane's row segment: destination and valid bytes (a multiple of 16)
      const int64_t e = e_unit + 256 * g + 128 * half;
      const int64_t nb = active ? (P.kp - e < 128 ? P.kp - e : 128) : 0;
      int8_t* dst = P.res + t * P.mod_stride + q * P.plane + int64_t(row) * P.kp + e;
      {
        // coalesced: per instruction 4 rows x 8 lanes x 16 bytes
        __syncwarp();
        const unsigned long long dst_u = reinterpret_cast<unsigned long long>(dst);
        const unsigned char* wst = St + b * TC_S_BYTES + uint32_t(quarter * 32) * TC_ROW_STAGE +
                                   uint32_t(half * 128);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int r = 4 * i + (lane >> 3), c = lane & 7;
          const unsigned long long rd = __shfl_sync(0xffffffffu, dst_u, r);
          const int64_t rn = __shfl_sync(0xffffffffu, nb, r);
          if (16 * c < rn)
            *reinterpret_cast<uint4*>(reinterpret_cast<int8_t*>(rd) + 16 * c) =
                *reinterpret_cast<const uint4*>(wst + r * TC_ROW_STAGE + 16 * c);
        }
        __syncwarp();
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0) atomicExch(P.status, 1);
  if (warp == 12) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem_base)
                 : "memory");
  }
}

// --------------------------------------------------------------------------
// 3. INT8 residue GEMM on tcgen05

struct GemmParams {
  int m;             // rows of A per product plane
  int nb;            // rows of B per product plane
  int kblocks;       // kp / 128
  int nchunks;       // ceil(kblocks / kChunkBlocks)
  int chunk_blocks;  // k-blocks per chunk: ceil(kblocks / nchunks) <= kChunkBlocks
  int nmod;          // products: moduli x nsub (the A/B/R planes in order)
  int nsub;          // products per modulus (3 complex, 1 real): modulus = product / nsub
  int t0;            // first product of this launch (units cover t0 ..)
  int tiles_m, tiles_n;
  int total_units;   // moduli of the launch * nchunks * tiles
  int* R;            // accumulated residues [nmod][nb][m] (int32), or
  unsigned char* R8; // with a single k-chunk: the residues as bytes (no accumulation)
  int* status;       // set to 1 when a bounded wait gave up
  const int* active; // CTA-pair kernel: list of tiles to compute (fill mode), or null = all
  int n_active;
  unsigned long long wait_limit_ns;  // bound on every barrier wait
  int stall_test;    // 1: the producer issues no copies (exercises the bounded waits)
  int p[kMaxModuli];
  int c16[kMaxModuli], off[kMaxModuli];  // division-free v mod p (mod_residue)
  unsigned M[kMaxModuli];
  int epi_split;     // CTA-pair kernel: epilogue warps per TMEM lane quarter (1 or 2)
};

struct Unit {
  int t, c, tm, tn;
};


// Tile raster within one (product, k-chunk): bands of kBandTiles row tiles,
// row tiles fastest within a band. The units in flight at one time cover a
// few row tiles of A and a few column tiles of B, so that each A tile is
// read from DRAM once even when A is much taller than L2 holds (a plain
// row-fastest order re-reads all of A once per column tile).
constexpr int kBandTiles = 8;
__host__ __device__ __forceinline__ void band_tile(int tile, int tiles_m, int tiles_n, int& tm,
                                                   int& tn) {
  const int band_units = kBandTiles * tiles_n;
  const int band = tile / band_units, r = tile - band * band_units;
  const int left = tiles_m - band * kBandTiles;
  const int rows = left < kBandTiles ? left : kBandTiles;
  tm = band * kBandTiles + r % rows;
  tn = r / rows;
}

__device__ __forceinline__ Unit decode_unit(int u, const GemmParams& g) {
  Unit r;
  const int tiles = g.tiles_m * g.tiles_n;
  const int tile = u % tiles;
  const int rest = u / tiles;
  band_tile(tile, g.tiles_m, g.tiles_n, r.tm, r.tn);
  r.c = rest % g.nchunks;
  r.t = g.t0 + rest / g.nchunks;
  return r;
}

__global__ void __launch_bounds__(GEMM_THREADS, 1)
    oz_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
            const __grid_constant__ GemmParams g) {
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte aligned base for the 128-byte swizzle atoms
  const uint32_t raw_addr = smem_u32(smem_raw);
  const uint32_t base = (raw_addr + 1023u) & ~1023u;
  unsigned char* base_ptr = smem_raw + (base - raw_addr);
  const uint32_t bar_base = base + STAGES * STAGE_BYTES;
  auto full_bar = [&](int s) { return bar_base + 8u * s; };
  auto empty_bar = [&](int s) { return bar_base + 8u * (STAGES + s); };
  auto accf_bar = [&](int b) { return bar_base + 8u * (2 * STAGES + b); };
  auto acce_bar = [&](int b) { return bar_base + 8u * (2 * STAGES + 2 + b); };
  const uint32_t drain_bar = bar_base + 8u * (2 * STAGES + 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base_ptr + STAGES * STAGE_BYTES + 256);
  volatile int* abort = reinterpret_cast<volatile int*>(base_ptr + STAGES * STAGE_BYTES + 264);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);
      mbar_init(acce_bar(b), 128);
    }
    mbar_init(drain_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     smem_u32(tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    int stage = 0;
    uint32_t phase = 0;
    bool ok = g.stall_test == 0;
    for (int u = blockIdx.x; u < g.total_units && ok; u += gridDim.x) {
      const Unit w = decode_unit(u, g);
      const int kb0 = w.c * g.chunk_blocks;
      const int kb1 = min(g.kblocks, kb0 + g.chunk_blocks);
      const int arow = w.t * g.m + w.tm * BM;
      const int brow = w.t * g.nb + w.tn * BN;
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort, g.wait_limit_ns)) {
          ok = false;
          break;
        }
        mbar_arrive_expect_tx(full_bar(stage), STAGE_BYTES);
        const uint32_t sa = base + stage * STAGE_BYTES;
        tma_load_2d(sa, &tmA, kb * BKB, arow, full_bar(stage));
        tma_load_2d(sa + A_STAGE, &tmB, kb * BKB, brow, full_bar(stage));
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
    if (!ok && g.stall_test == 0) {
      // let the copies already issued land before the shared memory goes away
      for (int s = 0; s < STAGES; ++s) {
        const unsigned long long t0 = globaltimer();
        while (!mbar_try_wait(full_bar(s), 0) && !mbar_try_wait(full_bar(s), 1) &&
               globaltimer() - t0 < 1000000ull) {
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    int stage = 0;
    uint32_t phase = 0;
    uint32_t acc_phase[2] = {0, 0};
    int accb = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < g.total_units && ok; u += gridDim.x) {
      const Unit w = decode_unit(u, g);
      const int kb0 = w.c * g.chunk_blocks;
      const int kb1 = min(g.kblocks, kb0 + g.chunk_blocks);
      if (!mbar_wait(acce_bar(accb), acc_phase[accb] ^ 1u, abort, g.wait_limit_ns)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t d = tmem_base + uint32_t(accb * BN);
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!mbar_wait(full_bar(stage), phase, abort, g.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = base + stage * STAGE_BYTES;
#pragma unroll
        for (int kk = 0; kk < BKB / 32; ++kk) {
          const uint64_t ad = umma_desc_sw128(sa + kk * 32);
          const uint64_t bd = umma_desc_sw128(sa + A_STAGE + kk * 32);
          umma_i8(d, ad, bd, (kb > kb0 || kk > 0) ? 1u : 0u);
        }
        umma_commit(empty_bar(stage));
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1u;
        }
      }
      if (!ok) break;
      umma_commit(accf_bar(accb));
      acc_phase[accb] ^= 1u;
      accb ^= 1;
    }
    if (!ok) {
      // MMAs may still be in flight: wait (bounded) until they retire
      umma_commit(drain_bar);
      const unsigned long long t0 = globaltimer();
      while (!mbar_try_wait(drain_bar, 0) && globaltimer() - t0 < 1000000ull) {
      }
    }
  } else if (warp >= 2) {
    // ---- epilogue: TMEM -> registers -> mod p -> accumulate into R
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
    const int row = quarter * 32 + lane;
    uint32_t acc_phase[2] = {0, 0};
    int accb = 0;
    for (int u = blockIdx.x; u < g.total_units; u += gridDim.x) {
      const Unit w = decode_unit(u, g);
      // warp-uniform: the TMEM loads below are collective
      if (!__all_sync(0xffffffffu,
                      mbar_wait(accf_bar(accb), acc_phase[accb], abort, g.wait_limit_ns)))
        break;
      tc_fence_after();
      const int mt = w.t / g.nsub;  // modulus of this product
      const int p = g.p[mt], c16 = g.c16[mt], off = g.off[mt];
      const unsigned M = g.M[mt];
      const int i = w.tm * BM + row;
      const int j0 = w.tn * BN;
      int* Rt = g.R + int64_t(w.t) * g.nb * g.m;
      for (int c0 = 0; c0 < BN; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tmem_base + (uint32_t(quarter * 32) << 16) + uint32_t(accb * BN + c0), v);
        if (i < g.m) {
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const int j = j0 + c0 + c;
            if (j < g.nb) {
              const int r = mod_residue(int(v[c]), p, c16, off, M);
              if (g.R8)
                g.R8[int64_t(w.t) * g.nb * g.m + int64_t(j) * g.m + i] = (unsigned char)r;
              else
                atomicAdd(Rt + int64_t(j) * g.m + i, r);
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acce_bar(accb));
      acc_phase[accb] ^= 1u;
      accb ^= 1;
    }
  }

  tc_fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0) atomicExch(g.status, 1);
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem_base)
                 : "memory");
  }
}

// --------------------------------------------------------------------------
// 3b. the same GEMM on CTA pairs (tcgen05 cta_group::2)
//
// A cluster of two CTAs computes a 256 x 256 tile: each CTA stages 128 rows of
// A and 128 rows of B per k-block (TMA, no multicast), the even CTA issues
// tcgen05.mma.cta_group::2 (M = 256, N = 256, K = 32) reading both CTAs'
// shared memory, and each CTA's TMEM receives its 128 rows of the tile. Per
// SM this halves the shared-memory operand traffic of the 1-CTA form and
// runs the tensor pipe at its full int8 rate.
//   full[s]  (even CTA): TMA bytes of both CTAs + the even producer's arrival
//   empty[s] (both):     commit of the MMAs, multicast to the pair
//   accf[b]  (both):     commit after a tile's last k-block, multicast
//   acce[b]  (even CTA): 256 epilogue threads of both CTAs, remote arrivals
// NT = 1: pair tile 256 x 256, two accumulator buffers (2 x 256 TMEM
// columns), 6 stages. NT = 2: pair tile 256 x 512 (two MMAs of N = 256 per
// k-step on one A tile: a quarter less L2 -> SMEM traffic per operation), one
// accumulator buffer of 512 columns (drained once per unit of 976 k-blocks),
// 4 stages.
constexpr int A_STAGE2 = 128 * BKB;  // 16 KiB per CTA
constexpr int B_HALF2 = 128 * BKB;   // 16 KiB per CTA and N = 256 half
template <int NT>
struct PairCfg {
  static constexpr int STAGES = NT == 1 ? 6 : 4;
  static constexpr int STAGE = A_STAGE2 + NT * B_HALF2;
  static constexpr int SMEM = STAGES * STAGE + 1024 + 1024;
  static constexpr int NBUF = NT == 1 ? 2 : 1;
};
constexpr uint32_t kIdescI8Pair = (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(256 >> 3) << 17) |
                                  (uint32_t(256 >> 4) << 24);

__device__ __forceinline__ void umma_i8_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                             uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescI8Pair), "r"(accumulate)
      : "memory");
}
// warp 0: TMA, warp 1: MMA, warps 2-9: epilogue. With g.epi_split = 2 two
// warps per TMEM lane quarter each drain half of the tile's columns: the
// per-value reduction is issue-bound, and one warp per scheduler made it the
// bottleneck when the units are short in k. With long units (the drain hides
// behind the next unit's MMAs) warps 2-5 drain alone and warps 6-9 idle.
constexpr int PAIR_THREADS = 320;
template <int NT>
__global__ void __launch_bounds__(PAIR_THREADS, 1)
    oz_gemm_pair(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ GemmParams g) {
  using P = PairCfg<NT>;
  constexpr int STAGES2 = P::STAGES;
  constexpr int STAGE2_BYTES = P::STAGE;
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  const uint32_t base = (raw_addr + 1023u) & ~1023u;
  unsigned char* base_ptr = smem_raw + (base - raw_addr);
  const uint32_t bar_base = base + STAGES2 * STAGE2_BYTES;
  auto full_bar = [&](int s) { return bar_base + 8u * s; };
  auto empty_bar = [&](int s) { return bar_base + 8u * (STAGES2 + s); };
  auto accf_bar = [&](int b) { return bar_base + 8u * (2 * STAGES2 + b); };
  auto acce_bar = [&](int b) { return bar_base + 8u * (2 * STAGES2 + 2 + b); };
  const uint32_t drain_bar = bar_base + 8u * (2 * STAGES2 + 4);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base_ptr + STAGES2 * STAGE2_BYTES + 256);
  volatile int* abort = reinterpret_cast<volatile int*>(base_ptr + STAGES2 * STAGE2_BYTES + 264);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();  // 0: issues the MMAs
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int tiles = g.tiles_m * g.tiles_n;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES2; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);
      mbar_init(acce_bar(b), 2 * 4 * g.epi_split);  // one arrival per epilogue warp of the pair
    }
    mbar_init(drain_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     smem_u32(tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const int ntl = g.active ? g.n_active : tiles;
  auto unit_of = [&](int u, int& t, int& c, int& tm, int& tn) {
    const int tl = u % ntl, rest = u / ntl;
    if (g.active) {  // explicit list: tm + tn * tiles_m
      const int tile = g.active[tl];
      tm = tile % g.tiles_m;
      tn = tile / g.tiles_m;
    } else {
      band_tile(tl, g.tiles_m, g.tiles_n, tm, tn);
    }
    c = rest % g.nchunks;
    t = g.t0 + rest / g.nchunks;
  };

  bool aborted = false;
  if (warp == 0 && lane == 0) {
    // ---- TMA producer (both CTAs): 128 rows of A and of B per k-block
    int stage = 0;
    uint32_t phase = 0;
    bool ok = g.stall_test == 0;
    for (int u = pair; u < g.total_units && ok; u += npairs) {
      int t, c, tm, tn;
      unit_of(u, t, c, tm, tn);
      const int kb0 = c * g.chunk_blocks, kb1 = min(g.kblocks, kb0 + g.chunk_blocks);
      const int arow = t * g.m + tm * 256 + int(rank) * 128;
      const int brow = t * g.nb + tn * (256 * NT) + int(rank) * 128;
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort, g.wait_limit_ns)) {
          ok = false;
          break;
        }
        const uint32_t fb = map_to_rank(full_bar(stage), 0);
        if (rank == 0) mbar_arrive_expect_tx(full_bar(stage), 2 * STAGE2_BYTES);
        const uint32_t sa = base + stage * STAGE2_BYTES;
        tma_load_2d_pair(sa, &tmA, kb * BKB, arow, fb);
#pragma unroll
        for (int h = 0; h < NT; ++h)
          tma_load_2d_pair(sa + A_STAGE2 + h * B_HALF2, &tmB, kb * BKB, brow + h * 256, fb);
        if (++stage == STAGES2) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
    aborted = !ok && g.stall_test == 0;
  } else if (warp == 1 && lane == 0 && rank == 0) {
    // ---- MMA issuer (even CTA)
    int stage = 0;
    uint32_t phase = 0;
    uint32_t acc_phase[2] = {0, 0};
    int accb = 0;
    bool ok = true;
    for (int u = pair; u < g.total_units && ok; u += npairs) {
      int t, c, tm, tn;
      unit_of(u, t, c, tm, tn);
      const int kb0 = c * g.chunk_blocks, kb1 = min(g.kblocks, kb0 + g.chunk_blocks);
      if (!mbar_wait(acce_bar(accb), acc_phase[accb] ^ 1u, abort, g.wait_limit_ns)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t d = tmem_base + uint32_t(accb * 256);
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!mbar_wait(full_bar(stage), phase, abort, g.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = base + stage * STAGE2_BYTES;
#pragma unroll
        for (int kk = 0; kk < BKB / 32; ++kk) {
          const uint64_t adesc = umma_desc_sw128(sa + kk * 32);
#pragma unroll
          for (int h = 0; h < NT; ++h)
            umma_i8_pair(d + uint32_t(h * 256),
                         adesc, umma_desc_sw128(sa + A_STAGE2 + h * B_HALF2 + kk * 32),
                         (kb > kb0 || kk > 0) ? 1u : 0u);
        }
        umma_commit_pair(empty_bar(stage));
        if (++stage == STAGES2) {
          stage = 0;
          phase ^= 1u;
        }
      }
      if (!ok) break;
      umma_commit_pair(accf_bar(accb));
      acc_phase[accb] ^= 1u;
      accb = (accb + 1) % P::NBUF;
    }
    if (!ok) {
      asm volatile(
          "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              drain_bar)
          : "memory");
      const unsigned long long t0 = globaltimer();
      while (!mbar_try_wait(drain_bar, 0) && globaltimer() - t0 < 1000000ull) {
      }
    }
  } else if (warp >= 2 && ((warp - 2) >> 2) < g.epi_split) {
    // ---- epilogue (both CTAs): own TMEM rows -> mod p -> R
    const int quarter = warp & 3;        // TMEM lanes 32*quarter .. +31
    const int half = (warp - 2) >> 2;    // columns half*kCols .. +kCols-1
    const int kCols = 256 * NT / g.epi_split;
    const int row = int(rank) * 128 + quarter * 32 + lane;
    uint32_t acc_phase[2] = {0, 0};
    int accb = 0;
    for (int u = pair; u < g.total_units; u += npairs) {
      int t, c, tm, tn;
      unit_of(u, t, c, tm, tn);
      // warp-uniform: the TMEM loads and the warp's arrival below are collective
      if (!__all_sync(0xffffffffu,
                      mbar_wait(accf_bar(accb), acc_phase[accb], abort, g.wait_limit_ns)))
        break;
      tc_fence_after();
      const int mt = t / g.nsub;  // modulus of this product
      const int p = g.p[mt], c16 = g.c16[mt], off = g.off[mt];
      const unsigned M = g.M[mt];
      const int i = tm * 256 + row;
      const int jw = tn * (256 * NT) + half * kCols;
      const int64_t plane = int64_t(t) * g.nb * g.m;
      for (int c0 = 0; c0 < kCols; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tmem_base + (uint32_t(quarter * 32) << 16) +
                      uint32_t(accb * 256 + half * kCols + c0),
                  v);
        const int jb = jw + c0;
        if (i < g.m && jb < g.nb) {
          const int64_t base = plane + int64_t(jb) * g.m + i;
          if (jb + 32 <= g.nb) {  // whole group of columns: no per-column test
            if (g.R8) {
              unsigned char* d = g.R8 + base;
#pragma unroll
              for (int cc = 0; cc < 32; ++cc)
                d[int64_t(cc) * g.m] = (unsigned char)mod_residue(int(v[cc]), p, c16, off, M);
            } else {
              int* d = g.R + base;
#pragma unroll
              for (int cc = 0; cc < 32; ++cc)
                atomicAdd(d + int64_t(cc) * g.m, mod_residue(int(v[cc]), p, c16, off, M));
            }
          } else {
#pragma unroll
            for (int cc = 0; cc < 32; ++cc) {
              if (jb + cc < g.nb) {
                const int r = mod_residue(int(v[cc]), p, c16, off, M);
                if (g.R8)
                  g.R8[base + int64_t(cc) * g.m] = (unsigned char)r;
                else
                  atomicAdd(g.R + base + int64_t(cc) * g.m, r);
              }
            }
          }
        }
      }
      // the accumulator is drained: one arrival per warp with the default
      // (CTA-scope) semantics on the MMA issuer's barrier; the ordering of the
      // TMEM loads before the next MMAs comes from the tcgen05 fences around
      // the barrier (a cluster-scope release per thread cost membar stalls)
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_remote(map_to_rank(acce_bar(accb), 0));
      acc_phase[accb] ^= 1u;
      accb = (accb + 1) % P::NBUF;
    }
  }

  if (aborted) {
    // copies issued by this CTA may still be landing in shared memory
    const unsigned long long t0 = globaltimer();
    while (globaltimer() - t0 < 2000000ull) {
    }
  }
  tc_fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0) atomicExch(g.status, 1);
  cluster_sync_all();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem_base)
                 : "memory");
  }
}

// --------------------------------------------------------------------------
// 4. reconstruction

constexpr long long kNaNBits = 0x7FF8000000000000ll;  // quiet NaN

// x * 2^e, correctly rounded: a multiplication by the power of two when the
// result stays normal (|x| is an integer below 2^128 or zero), ldexp otherwise.
__device__ __forceinline__ double scale_pow2(double x, int e) {
  if (e >= -1022 && e <= 895)
    return x * __longlong_as_double((long long)(e + 1023) << 52);
  return ldexp(x, e);
}

// C(i, j) <- alpha * x + beta * C(i, j) (x = xr + i xi for complex types)
template <int DT>
__device__ __forceinline__ void store_c(void* C, int64_t ci, double xr, double xi, double alr,
                                        double ali, double ber, double bei, bool read_c) {
  double outr = alr * xr - ali * xi, outi = alr * xi + ali * xr;
  if constexpr (DT == kC64) {
    double2* c = static_cast<double2*>(C) + ci;
    if (read_c) {
      const double2 old = *c;
      outr += ber * old.x - bei * old.y;
      outi += ber * old.y + bei * old.x;
    }
    *c = make_double2(outr, outi);
  } else if constexpr (DT == kC32) {
    float2* c = static_cast<float2*>(C) + ci;
    if (read_c) {
      const float2 old = *c;
      outr += ber * double(old.x) - bei * double(old.y);
      outi += ber * double(old.y) + bei * double(old.x);
    }
    *c = make_float2(float(outr), float(outi));
  } else if constexpr (DT == kR64) {
    double* c = static_cast<double*>(C) + ci;
    *c = read_c ? fma(ber, *c, outr) : outr;
  } else {
    float* c = static_cast<float*>(C) + ci;
    *c = float(read_c ? fma(ber, double(*c), outr) : outr);
  }
}

// Residues of element (i, j) of the real result (real types) or of Re and Im
// (complex: three product planes per modulus combined by combine3), for
// modulus t. src points at plane 0 of modulus t, element (i, j); planes of
// one product are `plane` elements apart. off: p for byte residues, off24 for
// int32 sums.
template <bool CPLX, typename RT>
__device__ __forceinline__ void product_residues(const RT* src, int64_t plane, int off, int conj,
                                                 int& re, int& im) {
  if (CPLX) {
    combine3(int(src[0]), int(src[plane]), int(src[2 * plane]), off, conj, re, im);
  } else {
    re = int(src[0]);
    im = 0;
  }
}

// C(i, j) <- alpha * 2^(-sigma_i - tau_j) * X + beta * C(i, j), X the CRT
// value of the product (complex: of Re and Im). R holds, per product plane,
// int32 sums of per-chunk residues or, with one k-chunk, the residues as
// bytes (RT). Threads run along i (contiguous in R and C), blocks along j: no
// index division. NM: the number of moduli when fixed at compile time (the
// defaults), 0 for rp.n.
template <int DT, typename RT, int NM>
__global__ void __launch_bounds__(256, 2) oz_reconstruct(const RT* __restrict__ R, int m, int n,
                                                         int nb, const int* __restrict__ sigA,
                                                         const int* __restrict__ sigB, void* C,
                                                         int64_t ldc, double alr, double ali,
                                                         double ber, double bei, int fill,
                                                         int64_t ro, int64_t co, int tile_m,
                                                         int tile_n, ReconParams rp) {
  constexpr bool CPLX = dtype_is_complex(DT);
  constexpr int NSUB = CPLX ? 3 : 1;
  constexpr bool kBytes = sizeof(RT) == 1;
  constexpr int NMAX = NM > 0 ? NM : kMaxUsableModuli;
  const int nmod = NM > 0 ? NM : rp.n;
  const int64_t plane = int64_t(nb) * m;
  const bool read_c = (ber != 0.0 || bei != 0.0);
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const int tauj = sigB[j];
    const int64_t tj = (j / tile_n) * int64_t(tile_n);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
      if (fill != 0) {
        const int64_t ti = (i / tile_m) * int64_t(tile_m);
        if (!tile_is_active(fill, ti, tj, ::min((int64_t)tile_m, (int64_t)m - ti),
                            ::min((int64_t)tile_n, (int64_t)n - tj), ro, co))
          continue;
      }
      int rr[NMAX], ri[NMAX];
      const RT* src = R + int64_t(j) * m + i;
#pragma unroll
      for (int t = 0; t < NMAX; ++t)
        if (t < nmod)
          product_residues<CPLX>(src + t * NSUB * plane, plane, kBytes ? rp.p[t] : rp.off24[t],
                                 rp.conj, rr[t], ri[t]);
      const int si = sigA[i];
      const int e = -(si + tauj);
      double xr = scale_pow2(crt_value<NM, kBytes>(rr, rp), e);
      double xi = CPLX ? scale_pow2(crt_value<NM, kBytes>(ri, rp), e) : 0.0;
      if (si == kSigmaNonFinite || tauj == kSigmaNonFinite) xr = xi = __longlong_as_double(kNaNBits);
      store_c<DT>(C, i + int64_t(j) * ldc, xr, xi, alr, ali, ber, bei, read_c);
    }
  }
}

// At(kk, i) <- A(i, kk): op(A) = N operands (A stored m-major) are copied
// k-major so that the row norms and the slicing read them like op(A) = T.
// 32 x 32 tiles through shared memory: reads run along i, writes along kk.
template <typename E>
__global__ void oz_transpose(const E* __restrict__ A, int64_t lda, int m, int64_t k,
                             E* __restrict__ At, int64_t ldat) {
  __shared__ E tile[32][33];
  const int i0 = blockIdx.x * 32;
  for (int64_t k0 = int64_t(blockIdx.y) * 32; k0 < k; k0 += int64_t(gridDim.y) * 32) {
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int i = i0 + threadIdx.x;
      const int64_t kk = k0 + r;
      if (i < m && kk < k) tile[r][threadIdx.x] = A[i + kk * lda];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      const int i = i0 + r;
      const int64_t kk = k0 + threadIdx.x;
      if (i < m && kk < k) At[int64_t(i) * ldat + kk] = tile[threadIdx.x][r];
    }
    __syncthreads();
  }
}

// The same reconstruction for byte residues with m % 16 == 0, staged through
// shared memory: a work item is one column j of C and a block of 1024 rows;
// its residues (moduli x product planes x 1024 bytes) are copied with 16-byte
// asynchronous copies into one of two stages while the previous item is
// reconstructed from the other, so that the CRT arithmetic does not wait on
// the loads. Items are spread over a grid of resident blocks (item =
// blockIdx.x + k * gridDim.x, row blocks fastest). Each thread takes four
// consecutive rows: byte q of word threadIdx.x of each 1024-byte plane.
constexpr int kStageRows = 1024;
template <int DT, int NM>
__global__ void __launch_bounds__(256, 2)
    oz_reconstruct_staged(const unsigned char* __restrict__ R, int m, int n, int nb,
                          const int* __restrict__ sigA, const int* __restrict__ sigB, void* C,
                          int64_t ldc, double alr, double ali, double ber, double bei, int fill,
                          int64_t ro, int64_t co, int tile_m, int tile_n, ReconParams rp) {
  constexpr bool CPLX = dtype_is_complex(DT);
  constexpr int NSUB = CPLX ? 3 : 1;
  constexpr int NMAX = NM > 0 ? NM : kMaxUsableModuli;
  constexpr int WPP = kStageRows / 4;  // 32-bit words per staged plane
  extern __shared__ uint4 stage_smem[];
  const int nmod = NM > 0 ? NM : rp.n;
  const int stage_words = NSUB * nmod * WPP;
  unsigned* stage = reinterpret_cast<unsigned*>(stage_smem);
  const int64_t plane = int64_t(nb) * m;
  const int row_blocks = (m + kStageRows - 1) / kStageRows;
  const int64_t items = int64_t(row_blocks) * n;
  const bool read_c = (ber != 0.0 || bei != 0.0);

  // staged plane pl = t * NSUB + s holds product s of modulus t
  auto prefetch = [&](int64_t item, int s) {
    const int rb = int(item % row_blocks), j = int(item / row_blocks);
    const int i0 = rb * kStageRows;
    const int chunks = min(kStageRows, m - i0) / 16;  // m % 16 == 0
    const int total = NSUB * nmod * chunks;
    unsigned* dst = stage + s * stage_words;
    for (int c = threadIdx.x; c < total; c += blockDim.x) {
      const int pl = c / chunks, ch = c - pl * chunks;
      const unsigned char* src = R + pl * plane + int64_t(j) * m + i0 + ch * 16;
      cp_async_16_cg(dst + pl * WPP + ch * 4, src);
    }
  };

  int64_t item = blockIdx.x;
  if (item < items) prefetch(item, 0);
  cp_async_commit();
  int s = 0;
  for (; item < items; item += gridDim.x) {
    const int64_t next = item + gridDim.x;
    if (next < items) prefetch(next, s ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int rb = int(item % row_blocks), j = int(item / row_blocks);
    const int i = rb * kStageRows + 4 * threadIdx.x;
    bool active = i < m;
    if (active && fill != 0) {  // tile_m is a multiple of 4: the four rows share a tile
      const int64_t ti = (i / tile_m) * int64_t(tile_m), tj = (j / tile_n) * int64_t(tile_n);
      active = tile_is_active(fill, ti, tj, ::min((int64_t)tile_m, (int64_t)m - ti),
                              ::min((int64_t)tile_n, (int64_t)n - tj), ro, co);
    }
    if (active) {
      const unsigned* w = stage + s * stage_words + threadIdx.x;
      const int tauj = sigB[j];
      // residues of Re (part 0) or Im (part 1) of row i + q, from the staged
      // bytes (the arrays of the two parts are built one after the other)
      auto part_residues = [&](int q, int part, int (&r)[NMAX]) {
#pragma unroll
        for (int t = 0; t < NMAX; ++t) {
          if (t < nmod) {
            const unsigned* wt = w + t * NSUB * WPP;
            const int r0 = int((wt[0] >> (8 * q)) & 255u);
            if (CPLX) {
              const int r1 = int((wt[WPP] >> (8 * q)) & 255u);
              const int r2 = int((wt[2 * WPP] >> (8 * q)) & 255u);
              int re, im;
              combine3(r0, r1, r2, rp.p[t], rp.conj, re, im);
              r[t] = part ? im : re;
            } else {
              r[t] = r0;
            }
          }
        }
      };
#pragma unroll 1
      for (int q = 0; q < 4; ++q) {  // rolled: one row's chain at a time keeps registers
        const int si = sigA[i + q];
        const int e = -(si + tauj);
        int r[NMAX];
        part_residues(q, 0, r);
        double xr = scale_pow2(crt_value<NM, true>(r, rp), e);
        double xi = 0.0;
        if (CPLX) {
          part_residues(q, 1, r);
          xi = scale_pow2(crt_value<NM, true>(r, rp), e);
        }
        if (si == kSigmaNonFinite || tauj == kSigmaNonFinite) xr = xi = __longlong_as_double(kNaNBits);
        store_c<DT>(C, i + q + int64_t(j) * ldc, xr, xi, alr, ali, ber, bei, read_c);
      }
    }
    __syncthreads();  // the stage is refilled by the next iteration's prefetch
    s ^= 1;
  }
  cp_async_wait<0>();
}

inline int staged_smem_bytes(bool cplx, int nmod) {
  return 2 * (cplx ? 3 : 1) * nmod * kStageRows;
}

// --------------------------------------------------------------------------
// 4b. CRT reconstruction on the tensor cores (byte residues, m % 16 == 0)
//
// By linearity the CRT sum needs no reduction of the product combination:
// with V_k the weight of product plane k, W_t for the plane's modulus t where
// the product enters Re or Im with a plus sign and P - W_t where it enters
// with a minus (Re = P0 -+ P1, Im = P2 - P0 -+ P1, see combine3; p_t W_t = 0
// mod P), S = sum_k r_k V_k is congruent mod P to the sum the CUDA-core
// kernels form. Written in the bytes of V_k, S = sum_j 256^j S_j with
// S_j = sum_k r_k byte_j(V_k), and for 128 consecutive rows of one column of
// C one tcgen05.mma kind::i8 (unsigned bytes, exact INT32 sums below 2^22)
//   D[128 x NO] = R[128 x KP] . V[KP x NO]
// forms all of them: R is the tile's residue bytes as TMA loads them (one
// 128-byte row per product plane: the MN-major operand layout), V the
// weight bytes (K-major, columns 0-15 for Re, 16-31 for Im). The epilogue
// (one TMEM lane per row of C) combines its 16 sums per part into the four
// 32-bit limb sums of S and finishes with crt_from_limbs, as the CUDA-core
// kernels do: the results are the same doubles.
//
// A work unit is RT_G blocks of 128 rows of one column (the fixed cost of the
// hand-offs below is paid once per unit). Warp 0: TMA producer (4-stage
// ring), warp 1: TMEM allocation and MMA issue (accumulators double-buffered),
// warps 2-5: epilogue (RT_G rows per lane). Every wait is bounded; a give-up
// sets *status.
constexpr int RT_THREADS = 192;
constexpr int RT_STAGES = 4;
constexpr int RT_G = 2;                       // blocks of 128 rows per work unit
constexpr int RT_KP = 64;                     // planes per block (K), padded
constexpr int RT_BLOCK = 128 * RT_KP;         // bytes per block of 128 rows
constexpr int RT_STAGE = RT_G * RT_BLOCK;     // bytes per stage
constexpr int RT_W_BYTES = 32 * 128;          // weights: 32 rows x 128 B (SW128)
constexpr int RT_SMEM = RT_STAGES * RT_STAGE + RT_W_BYTES + 256 + 1024;
// three CTAs fit an SM's shared memory, so their 2 x RT_G x 32 TMEM columns fit
static_assert(4 * (RT_SMEM + 1024) > 228 * 1024 && 3 * 2 * RT_G * 32 <= 512,
              "at most three CTAs per SM, within the TMEM");

struct ReconTcParams {
  int m, n;
  int row_blocks;         // groups of RT_G blocks of 128 rows: ceil(m / (128 RT_G))
  long long total_units;  // row_blocks * n
  int planes;             // product planes of the residue array (loaded per tile)
  int kp;                 // K of the MMA: 32 or 64 (planes past `planes` are zero rows)
  const int* sigA;
  const int* sigB;
  void* C;
  int64_t ldc;
  double alr, ali, ber, bei;
  int fill;
  int64_t ro, co;
  int tile_m, tile_n;
  ReconParams rp;
  unsigned char v[32][RT_KP];  // weight bytes: v[o][k] = byte (o % 16) of V_k for part o / 16
  int* status;
  unsigned long long wait_limit_ns;
};

// UMMA shared-memory descriptor of an MN-major operand in the 128-byte
// swizzle layout: 8-row atoms of 128 bytes along M (one atom covers the 128
// rows of the tile), atoms 1024 B apart along K.
__device__ __forceinline__ uint64_t umma_desc_sw128_mn(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);  // start address
  d |= uint64_t(1) << 16;                  // leading byte offset (one atom along M: unused)
  d |= uint64_t(1024 >> 4) << 32;          // stride byte offset: 8 K-rows x 128 B
  d |= uint64_t(1) << 46;                  // descriptor version (sm_100)
  d |= uint64_t(2) << 61;                  // layout: 128-byte swizzle
  return d;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

template <int DT>
__global__ void __launch_bounds__(RT_THREADS, 3)
    oz_reconstruct_tc(const __grid_constant__ CUtensorMap tmR,
                      const __grid_constant__ ReconTcParams P) {
  constexpr bool CPLX = dtype_is_complex(DT);
  constexpr int NO = CPLX ? 32 : 16;  // output columns of the MMA
  // D S32, A and B unsigned int8, A MN-major, B K-major, N = NO, M = 128
  constexpr uint32_t kIdesc = (2u << 4) | (1u << 15) | (uint32_t(NO >> 3) << 17) |
                              (uint32_t(128 >> 4) << 24);
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw_addr = smem_u32(smem_raw);
  const uint32_t base = (raw_addr + 1023u) & ~1023u;
  unsigned char* base_ptr = smem_raw + (base - raw_addr);
  const uint32_t w_addr = base + RT_STAGES * RT_STAGE;
  const uint32_t bar_base = w_addr + RT_W_BYTES;
  auto full_bar = [&](int s) { return bar_base + 8u * s; };
  auto empty_bar = [&](int s) { return bar_base + 8u * (RT_STAGES + s); };
  auto accf_bar = [&](int b) { return bar_base + 8u * (2 * RT_STAGES + b); };
  auto acce_bar = [&](int b) { return bar_base + 8u * (2 * RT_STAGES + 2 + b); };
  const uint32_t drain_bar = bar_base + 8u * (2 * RT_STAGES + 4);
  unsigned char* ctl = base_ptr + RT_STAGES * RT_STAGE + RT_W_BYTES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ctl + 8 * (2 * RT_STAGES + 5));
  volatile int* abort = reinterpret_cast<volatile int*>(ctl + 8 * (2 * RT_STAGES + 5) + 8);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // weight bytes into the K-major 128-byte-swizzled B tile (row o, K byte k),
  // and zeros into the plane rows planes .. kp-1 of every stage (TMA writes
  // rows 0 .. planes-1 only)
  {
    unsigned char* wp = base_ptr + RT_STAGES * RT_STAGE;
    for (int idx = threadIdx.x; idx < RT_W_BYTES; idx += RT_THREADS) {
      const int o = idx >> 7, k = idx & 127;
      const unsigned char b = (o < NO && k < P.kp) ? P.v[o][k] : 0;
      wp[(o >> 3) * 1024 + (o & 7) * 128 + (((k >> 4) ^ (o & 7)) << 4) + (k & 15)] = b;
    }
    const int pad = (P.kp - P.planes) * 128;  // bytes per block, 16-byte words below
    for (int idx = threadIdx.x; idx < RT_STAGES * RT_G * (pad / 16); idx += RT_THREADS) {
      const int blk = idx / (pad / 16), w16 = idx - blk * (pad / 16);  // blk: stage, block
      *reinterpret_cast<uint4*>(base_ptr + blk * RT_BLOCK + P.planes * 128 + 16 * w16) =
          make_uint4(0u, 0u, 0u, 0u);
    }
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < RT_STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);
      mbar_init(acce_bar(b), 4);
    }
    mbar_init(drain_bar, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // the tensor cores read the weights through the async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)), "n"(2 * RT_G * 32)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t tile_bytes = uint32_t(RT_G * 128 * P.planes);
  bool copies_pending = false;  // the producer gave up with copies possibly in flight

  // unit u = (row block rb, column j), u = rb + j row_blocks: every role walks
  // u = blockIdx.x, + gridDim.x, ... with (rb, j) advanced without division
  const int drb = int(gridDim.x % unsigned(P.row_blocks));
  const int dj = int(gridDim.x / unsigned(P.row_blocks));
  auto next_unit = [&](int& rb, int& j) {
    rb += drb;
    j += dj;
    if (rb >= P.row_blocks) {
      rb -= P.row_blocks;
      ++j;
    }
  };
  const int rb0 = int(blockIdx.x % unsigned(P.row_blocks));
  const int j0 = int(blockIdx.x / unsigned(P.row_blocks));

  if (warp == 0 && lane == 0) {
    // ---- TMA producer: the tile's planes, 128 residue bytes each
    int rb = rb0, j = j0;
    for (long long u = blockIdx.x, it = 0; u < P.total_units;
         u += gridDim.x, ++it, next_unit(rb, j)) {
      const int stage = int(it % RT_STAGES);
      const uint32_t phase = uint32_t((it / RT_STAGES) & 1);
      if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort, P.wait_limit_ns)) {
        copies_pending = true;
        break;
      }
      mbar_arrive_expect_tx(full_bar(stage), tile_bytes);
      // the last group's blocks past m read as zeros (their rows are not stored)
#pragma unroll
      for (int g = 0; g < RT_G; ++g)
        tma_load_3d(base + stage * RT_STAGE + g * RT_BLOCK, &tmR, (rb * RT_G + g) * 128, j, 0,
                    full_bar(stage));
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    bool ok = true;
    for (long long u = blockIdx.x, it = 0; u < P.total_units; u += gridDim.x, ++it) {
      const int stage = int(it % RT_STAGES);
      const uint32_t phase = uint32_t((it / RT_STAGES) & 1);
      const int b = int(it & 1);
      const uint32_t bpar = uint32_t((it >> 1) & 1);
      if (!mbar_wait(acce_bar(b), bpar ^ 1u, abort, P.wait_limit_ns) ||
          !mbar_wait(full_bar(stage), phase, abort, P.wait_limit_ns)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t sa = base + stage * RT_STAGE;
#pragma unroll
      for (int g = 0; g < RT_G; ++g)
        for (int kb = 0; kb < P.kp / 32; ++kb)
          umma_i8_desc(tmem_base + uint32_t((b * RT_G + g) * 32),
                       umma_desc_sw128_mn(sa + g * RT_BLOCK + kb * 4096),
                       umma_desc_sw128(w_addr + kb * 32), kIdesc, kb > 0 ? 1u : 0u);
      umma_commit(empty_bar(stage));
      umma_commit(accf_bar(b));
    }
    if (!ok) {
      umma_commit(drain_bar);  // MMAs may be in flight: wait (bounded) until they retire
      const unsigned long long t0 = globaltimer();
      while (!mbar_try_wait(drain_bar, 0) && globaltimer() - t0 < 1000000ull) {
      }
    }
  } else if (warp >= 2) {
    // ---- epilogue: lane quarter (warp % 4), one row of C per lane
    const int quarter = warp & 3;
    const bool read_c = (P.ber != 0.0 || P.bei != 0.0);
    const uint32_t lane_taddr = tmem_base + (uint32_t(quarter * 32) << 16);
    int rb = rb0, j = j0;
    for (long long u = blockIdx.x, it = 0; u < P.total_units;
         u += gridDim.x, ++it, next_unit(rb, j)) {
      const int b = int(it & 1);
      const uint32_t bpar = uint32_t((it >> 1) & 1);
      // the scale exponents load while the accumulator is awaited
      int si[RT_G];
#pragma unroll
      for (int g = 0; g < RT_G; ++g) {
        const int i = (rb * RT_G + g) * 128 + quarter * 32 + lane;
        si[g] = i < P.m ? P.sigA[i] : 0;
      }
      const int tauj = P.sigB[j];
      // warp-uniform: the TMEM loads and the warp's arrival below are collective
      if (!__all_sync(0xffffffffu, mbar_wait(accf_bar(b), bpar, abort, P.wait_limit_ns))) break;
      tc_fence_after();
      __syncwarp();
      uint32_t v[RT_G][32];
#pragma unroll
      for (int g = 0; g < RT_G; ++g)
        tmem_ld32_nowait(lane_taddr + uint32_t((b * RT_G + g) * 32), v[g]);
      tmem_wait_ld();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce_bar(b));  // the accumulator may be overwritten
#pragma unroll
      for (int g = 0; g < RT_G; ++g) {
        const int i = (rb * RT_G + g) * 128 + quarter * 32 + lane;
        bool active = i < P.m;
        if (active && P.fill != 0) {
          const int64_t ti = (i / P.tile_m) * int64_t(P.tile_m);
          const int64_t tj = (j / P.tile_n) * int64_t(P.tile_n);
          active = tile_is_active(P.fill, ti, tj, ::min((int64_t)P.tile_m, (int64_t)P.m - ti),
                                  ::min((int64_t)P.tile_n, (int64_t)P.n - tj), P.ro, P.co);
        }
        if (active) {
          // limb L of S = sum of S_j 2^(8 (j - 4L)) over j = 4L .. 4L + 3 (below
          // 2^47): two 32-bit shift-adds (each below 2^31) and one wide multiply-add
          auto limb = [&](int j0) {
            const uint32_t a = v[g][j0] + (v[g][j0 + 1] << 8);
            const uint32_t bb = v[g][j0 + 2] + (v[g][j0 + 3] << 8);
            return (unsigned long long)bb * 65536ull + a;
          };
          const int e = -(si[g] + tauj);
          double xr =
              scale_pow2(crt_from_limbs<true>(limb(0), limb(4), limb(8), limb(12), P.rp), e);
          double xi = 0.0;
          if (CPLX)
            xi = scale_pow2(crt_from_limbs<true>(limb(16), limb(20), limb(24), limb(28), P.rp),
                            e);
          if (si[g] == kSigmaNonFinite || tauj == kSigmaNonFinite)
            xr = xi = __longlong_as_double(kNaNBits);
          store_c<DT>(P.C, i + int64_t(j) * P.ldc, xr, xi, P.alr, P.ali, P.ber, P.bei, read_c);
        }
      }
    }
  }

  if (copies_pending) {
    // copies issued by this CTA may still be landing in shared memory
    const unsigned long long t0 = globaltimer();
    while (globaltimer() - t0 < 2000000ull) {
    }
  }
  tc_fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0) atomicExch(P.status, 1);
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                 "n"(2 * RT_G * 32)
                 : "memory");
  }
}

// --------------------------------------------------------------------------
// host orchestration

struct Layout {
  int nmod;
  int nsub;                // products per modulus: 3 (complex, Karatsuba) or 1 (real)
  int64_t K2, kp;          // reals per operand row; residue row length (k padded to 128)
  int rowsA, rowsB, nb;    // A rows, B rows, B residue rows per product
  bool at;                 // op(A) = N too long for in-place tiles: A copied k-major
  bool mn;                 // op(A) = N: A read in place (m-major)
  bool mnB;                // op(B) = T or C: B read in place (n-major)
  int ksA, ksB;            // k-slices of the in-place row norms of A and B (1: none)
  bool r8;                 // one k-chunk: the residues of C are stored as bytes
  int64_t ldAt;            // leading dimension of At (elements of A's type)
  size_t off_sigA, off_sigB, off_resA, off_resB, off_R, off_At, off_status, off_tiles;
  size_t off_partA, off_partB;  // k-slice partial sums of the in-place row norms
  size_t off_ssq, off_list;     // one-pass row scaling (onepass_operands): scaled sums
                                // of squares, rows sent back and their two counts
  size_t total;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// In-place reading of an m-major operand: the transposing slicer's tiles of
// 128 (complex) or 256 (real) elements along k must fit the grid's y extent.
bool mn_fits(const GemmProblem& p) {
  const int64_t kp = (p.k + BKB - 1) / BKB * BKB;
  const int64_t kt = dtype_is_complex(p.dtype) ? 128 : 256;
  return (kp + kt - 1) / kt <= 65535;
}

// k-slices of the in-place row norms: about 2^18 threads in all (one per row
// and slice), slices of at least 512 elements, at most 4096 slices (the grid's
// y extent)
int norm_slices(int64_t rows, int64_t k) {
  if (rows >= kMnRows || k <= 512) return 1;
  const int64_t want = std::min<int64_t>(((int64_t(1) << 18) + rows - 1) / rows, 4096);
  return int(std::max<int64_t>(1, std::min<int64_t>(want, (k + 511) / 512)));
}

Layout layout_of(const GemmProblem& p, int moduli) {
  Layout L{};
  L.nmod = moduli > 0 ? std::min(moduli, kMaxUsableModuli)
                      : (dtype_is_double(p.dtype) ? kDefaultModuli : kDefaultModuliFloat);
  const bool cplx = dtype_is_complex(p.dtype);
  L.nsub = cplx ? 3 : 1;
  L.K2 = cplx ? 2 * p.k : p.k;
  L.kp = (p.k + BKB - 1) / BKB * BKB;
  L.rowsA = int(p.m);
  L.rowsB = int(p.n);
  L.nb = int(p.n);
  // op(A) = N and op(B) = T, C: read in place (the tiles of the transposing
  // slicer fit the grid), else A is copied k-major (B is then unsupported)
  L.mn = p.opA == 0 && mn_fits(p);
  L.at = p.opA == 0 && !L.mn;
  L.mnB = p.opB != 0;
  L.ksA = L.mn ? norm_slices(p.m, p.k) : 1;
  L.ksB = L.mnB ? norm_slices(p.n, p.k) : 1;
  L.r8 = (L.kp / BKB + kChunkBlocks - 1) / kChunkBlocks == 1;
  L.ldAt = L.at ? (p.k + 7) / 8 * 8 : 0;
  size_t off = 0;
  L.off_sigA = off;
  off = align256(off + sizeof(int) * L.rowsA);
  L.off_sigB = off;
  off = align256(off + sizeof(int) * L.rowsB);
  L.off_resA = off;
  off = align256(off + size_t(L.nmod) * L.nsub * L.rowsA * L.kp);
  L.off_resB = off;
  off = align256(off + size_t(L.nmod) * L.nsub * L.nb * L.kp);
  L.off_R = off;
  off = align256(off + (L.r8 ? 1 : sizeof(int)) * size_t(L.nmod) * L.nsub * L.nb * L.rowsA);
  L.off_At = off;
  off = align256(off + size_t(dtype_bytes(p.dtype)) * size_t(L.rowsA) * size_t(L.ldAt));
  L.off_status = off;
  off = align256(off + 256);
  L.off_tiles = off;
  off = align256(off + sizeof(int) * size_t((L.rowsA + 255) / 256) * ((L.nb + 255) / 256));
  L.off_partA = off;
  off = align256(off + (L.ksA > 1 ? size_t(L.ksA) * L.rowsA * (sizeof(double) + sizeof(int)) : 0));
  L.off_partB = off;
  off = align256(off + (L.ksB > 1 ? size_t(L.ksB) * L.rowsB * (sizeof(double) + sizeof(int)) : 0));
  L.off_ssq = off;  // A's rows, then B's
  off = align256(off + sizeof(double) * (size_t(L.rowsA) + L.rowsB));
  L.off_list = off;  // lists of A's and B's rows, their exact flags, the two counts
  off = align256(off + sizeof(int) * (2 * (size_t(L.rowsA) + L.rowsB) + 2));
  L.total = off;
  return L;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

bool make_map(CUtensorMap* map, void* base, int64_t kp, int64_t rows, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {cuuint64_t(kp), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(kp)};
  cuuint32_t box[2] = {cuuint32_t(BKB), cuuint32_t(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Residue bytes of C for the tensor-core reconstruction: dims (m, nb, planes)
// with strides (m, nb m) bytes (m % 16 == 0, m >= 128), boxes of 128 rows x 1
// column x all planes (rows past m read as zeros), 128-byte swizzle: one
// 128-byte row per plane, the MN-major operand layout.
bool make_map_recon(CUtensorMap* map, void* base, int m, int nb, int planes) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {cuuint64_t(m), cuuint64_t(nb), cuuint64_t(planes)};
  cuuint64_t strides[2] = {cuuint64_t(m), cuuint64_t(int64_t(nb) * m)};
  cuuint32_t box[3] = {128u, 1u, cuuint32_t(planes)};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

int sm_count() {
  int dev = 0, v = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v;
}

}  // namespace oz

size_t ozaki_workspace_bytes(const GemmProblem& p, int moduli) {
  if (p.m <= 0 || p.n <= 0) return 0;
  return oz::layout_of(p, moduli).total;
}

bool ozaki_copies_a(const GemmProblem& p) { return p.opA == 0 && !oz::mn_fits(p); }

bool ozaki_supported(const GemmProblem& p) {
  // op(B) = T or C: B is read in place, which needs the slicer's tiles to fit
  return (p.opB == 0 || ((p.opB == 1 || p.opB == 2) && oz::mn_fits(p))) &&
         p.m <= (1 << 24) && p.n <= (1 << 23);
}

namespace {
// Reals per slicing thread: 8 by default (more resident warps), 16 with
// SPLAB_OZAKI_SLICE_EL=16.
int slice_elems() {
  static const int el = [] {
    const char* v = std::getenv("SPLAB_OZAKI_SLICE_EL");
    return (v && std::atoi(v) == 16) ? 16 : 8;
  }();
  return el;
}

// The default modulus count of the input type (15 for double, 9 for float)
// over all moduli runs unrolled (SPLAB_OZAKI_SLICE_UNROLL=0 keeps the loop).
bool slice_unroll() {
  static const bool on = [] {
    const char* v = std::getenv("SPLAB_OZAKI_SLICE_UNROLL");
    return !(v && v[0] == '0');
  }();
  return on;
}

template <typename TIn, bool VEC, int EL, int MODE>
void launch_slice_el(int ndig, unsigned grid, cudaStream_t st, const TIn* X, int64_t ld,
                     int64_t len, int rows, int64_t kp, const int* sig, int s_sign, int8_t* res,
                     int64_t stride, const oz::SliceConsts& sc, int t0, int t1, double* ssq) {
  using namespace oz;
  constexpr int kNU = sizeof(TIn) == 8 ? kDefaultModuli : kDefaultModuliFloat;
  constexpr int kDigU = sizeof(TIn) == 8 ? 4 : 3;  // digits of the default scaling
  if (t0 == 0 && t1 == kNU && sc.n == kNU && ndig == kDigU && slice_unroll()) {
    if (ssq)
      oz_slice<TIn, VEC, kDigU, EL, kNU, MODE, true><<<grid, 256, 0, st>>>(
          X, ld, len, rows, kp, sig, s_sign, res, stride, sc, t0, t1, ssq);
    else
      oz_slice<TIn, VEC, kDigU, EL, kNU, MODE><<<grid, 256, 0, st>>>(
          X, ld, len, rows, kp, sig, s_sign, res, stride, sc, t0, t1, nullptr);
    return;
  }
  if (ndig <= 3)
    oz_slice<TIn, VEC, 3, EL, 0, MODE><<<grid, 256, 0, st>>>(
        X, ld, len, rows, kp, sig, s_sign, res, stride, sc, t0, t1, nullptr);
  else if (ndig == 4)
    oz_slice<TIn, VEC, 4, EL, 0, MODE><<<grid, 256, 0, st>>>(
        X, ld, len, rows, kp, sig, s_sign, res, stride, sc, t0, t1, nullptr);
  else
    oz_slice<TIn, VEC, 5, EL, 0, MODE><<<grid, 256, 0, st>>>(
        X, ld, len, rows, kp, sig, s_sign, res, stride, sc, t0, t1, nullptr);
}

// ssq (unrolled default scaling only): also the rows' scaled sums of squares
template <typename TIn, bool VEC>
void launch_slice(int ndig, cudaStream_t st, const TIn* X, int64_t ld, int64_t len, int rows,
                  int64_t kp, const int* sig, int mode, int s_sign, int8_t* res, int64_t stride,
                  const oz::SliceConsts& sc, int t0, int t1, double* ssq = nullptr) {
  const int el = slice_elems();
  const int64_t kreal = mode == 2 ? 2 * kp : kp;  // reals per row a thread group covers
  const unsigned grid = unsigned((int64_t(rows) * (kreal / el) + 255) / 256);
  auto run = [&](auto el_tag, auto mode_tag) {
    launch_slice_el<TIn, VEC, decltype(el_tag)::value, decltype(mode_tag)::value>(
        ndig, grid, st, X, ld, len, rows, kp, sig, s_sign, res, stride, sc, t0, t1, ssq);
  };
  using E8 = std::integral_constant<int, 8>;
  using E16 = std::integral_constant<int, 16>;
  using M0 = std::integral_constant<int, 0>;
  using M2 = std::integral_constant<int, 2>;
  if (el == 16) {
    if (mode == 2) run(E16{}, M2{});
    else run(E16{}, M0{});
  } else {
    if (mode == 2) run(E8{}, M2{});
    else run(E8{}, M0{});
  }
}

// Residues of m-major rows (op(A) = N read in place): oz_slice_mn
template <typename TIn, bool VEC, int MODE>
void launch_slice_mn_v(int ndig, dim3 grid, cudaStream_t st, const TIn* X, int64_t ld, int m,
                       int64_t k, int64_t kp, const int* sig, int s_sign, int conj, int8_t* res,
                       int64_t stride, const oz::SliceConsts& sc, int t0, int t1) {
  using namespace oz;
  constexpr int kNU = sizeof(TIn) == 8 ? kDefaultModuli : kDefaultModuliFloat;
  constexpr int kDigU = sizeof(TIn) == 8 ? 4 : 3;
  if (t0 == 0 && t1 == kNU && sc.n == kNU && ndig == kDigU && slice_unroll()) {
    oz_slice_mn<TIn, VEC, kDigU, kNU, MODE>
        <<<grid, 256, 0, st>>>(X, ld, m, k, kp, sig, s_sign, conj, res, stride, sc, t0, t1);
    return;
  }
  if (ndig <= 3)
    oz_slice_mn<TIn, VEC, 3, 0, MODE>
        <<<grid, 256, 0, st>>>(X, ld, m, k, kp, sig, s_sign, conj, res, stride, sc, t0, t1);
  else if (ndig == 4)
    oz_slice_mn<TIn, VEC, 4, 0, MODE>
        <<<grid, 256, 0, st>>>(X, ld, m, k, kp, sig, s_sign, conj, res, stride, sc, t0, t1);
  else
    oz_slice_mn<TIn, VEC, 5, 0, MODE>
        <<<grid, 256, 0, st>>>(X, ld, m, k, kp, sig, s_sign, conj, res, stride, sc, t0, t1);
}

template <typename TIn>
void launch_slice_mn(int ndig, cudaStream_t st, const TIn* X, int64_t ld, int m, int64_t k,
                     int64_t kp, const int* sig, int mode, int s_sign, int conj, int8_t* res,
                     int64_t stride, const oz::SliceConsts& sc, int t0, int t1) {
  const int64_t kt = mode == 2 ? 128 : 256;  // elements per row per tile
  const dim3 grid(unsigned((m + 7) / 8), unsigned((kp + kt - 1) / kt));
  if (mode == 2) {
    // 16-byte element loads for complex double with a 16-byte aligned base
    if (sizeof(TIn) == 8 && reinterpret_cast<uintptr_t>(X) % 16 == 0)
      launch_slice_mn_v<TIn, true, 2>(ndig, grid, st, X, ld, m, k, kp, sig, s_sign, conj, res,
                                      stride, sc, t0, t1);
    else
      launch_slice_mn_v<TIn, false, 2>(ndig, grid, st, X, ld, m, k, kp, sig, s_sign, conj, res,
                                       stride, sc, t0, t1);
  } else {
    launch_slice_mn_v<TIn, false, 0>(ndig, grid, st, X, ld, m, k, kp, sig, s_sign, conj, res,
                                     stride, sc, t0, t1);
  }
}

// Row scale exponents of A (which & 1) and B (which & 2).
template <typename TIn>
void scale_operands(const oz::Layout& L, const oz::Crt& crt, const GemmProblem& p, bool cplx,
                    int* sigA, int* sigB, char* w, int which, cudaStream_t st) {
  using namespace oz;
  const int64_t ldA = cplx ? 2 * p.lda : p.lda;  // in real elements
  const int64_t ldB = cplx ? 2 * p.ldb : p.ldb;
  // m-major rows read in place: k-sliced norms, combined when sliced
  auto in_place = [&](const void* X, int64_t ld, int rows, int ks, size_t off_part, int* sig) {
    const int64_t kspan = (p.k + ks - 1) / ks;
    double* partS = reinterpret_cast<double*>(w + off_part);
    int* partE = reinterpret_cast<int*>(w + off_part + sizeof(double) * size_t(ks) * rows);
    const dim3 grid(unsigned((rows + 255) / 256), unsigned(ks));
    if (cplx)
      oz_row_scale_mn<TIn, true><<<grid, 256, 0, st>>>(static_cast<const TIn*>(X), ld, rows, p.k,
                                                       kspan, crt.q_bits, sig, partS, partE);
    else
      oz_row_scale_mn<TIn, false><<<grid, 256, 0, st>>>(static_cast<const TIn*>(X), ld, rows, p.k,
                                                        kspan, crt.q_bits, sig, partS, partE);
    if (ks > 1)
      oz_row_scale_combine<<<unsigned((rows + 255) / 256), 256, 0, st>>>(partS, partE, rows, ks,
                                                                         crt.q_bits, sig);
  };
  if ((which & 1) && L.mn)
    in_place(p.A, p.lda, L.rowsA, L.ksA, L.off_partA, sigA);
  else if (which & 1)
    oz_row_scale<TIn><<<L.rowsA, 256, 0, st>>>(static_cast<const TIn*>(p.A), ldA, L.K2,
                                               L.rowsA, crt.q_bits, sigA);
  if ((which & 2) && L.mnB)
    in_place(p.B, p.ldb, L.rowsB, L.ksB, L.off_partB, sigB);
  else if (which & 2)
    oz_row_scale<TIn><<<L.rowsB, 256, 0, st>>>(static_cast<const TIn*>(p.B), ldB, L.K2,
                                               L.rowsB, crt.q_bits, sigB);
}

// Residue slicing of complex double rows with the digit sums on the tensor
// cores (oz_slice_tc), selected by SPLAB_OZAKI_SLICE_TC=1 (read per call, so
// that tests compare both slicers in one process); used for all moduli at once
// when the modulus 256 comes first and the rows are 16-byte aligned. The FP32
// digit-sum slicer (oz_slice) is the default: on B200 it measured faster
// (headline problem: 5.25 + 4.75 ms against 5.77 + 5.10 ms for the residues
// of A and B), the tensor-core form being bound by instruction issue and
// latency (TMEM round trip, staging, synchronisation) rather than by the FP32
// pipe it relieves.
bool slice_tc_enabled() {
  const char* v = std::getenv("SPLAB_OZAKI_SLICE_TC");
  return v && v[0] == '1';
}

cudaError_t launch_slice_tc(const double* X, int64_t ld, int64_t len, int rows, int64_t kp,
                            const int* sig, int s_sum, int8_t* res, int64_t mod_stride,
                            int64_t plane, const oz::Crt& crt, int nmod, int* status,
                            cudaStream_t st) {
  using namespace oz;
  SliceTcParams P{};
  P.X = X;
  P.ld = ld;
  P.len = len;
  P.rows = rows;
  P.kp = kp;
  P.sigma = sig;
  P.s_sum = s_sum;
  P.res = res;
  P.mod_stride = mod_stride;
  P.plane = plane;
  P.nmod = nmod;
  const int r3 = 3 * (nmod - 1);
  P.groups = std::min(4, 128 / r3);
  P.ksteps = (16 * P.groups + 31) / 32;
  P.units_per_row = int((kp + 256 * P.groups - 1) / (256 * P.groups));
  P.total_units = (long long)rows * P.units_per_row;
  for (int t = 0; t < nmod; ++t) P.p[t] = crt.p[t];
  P.status = status;
  P.wait_limit_ns = kWaitLimitNs;
  if (P.total_units <= 0) return cudaSuccess;
  cudaError_t e = set_dynamic_smem(reinterpret_cast<const void*>(oz_slice_tc), TC_SMEM);
  if (e != cudaSuccess) return e;
  const long long grid = std::min<long long>(P.total_units, sm_count());
  oz_slice_tc<<<unsigned(grid), TC_THREADS, TC_SMEM, st>>>(P);
  return cudaGetLastError();
}

// Slicer constants of the moduli, and the digit count covering |x| <= 2^Q:
// 3 of 13 bits, 4 balanced of 15 bits, or 5 of 13.
oz::SliceConsts slice_consts(const oz::Layout& L, const oz::Crt& crt, int* ndig_out) {
  using namespace oz;
  SliceConsts sc{};
  sc.n = L.nmod;
  sc.p0 = float(crt.p[0]);
  for (int t = 0; t < L.nmod; ++t) {
    const int pt = crt.p[t];
    sc.neg_p[t] = f2_pack(-float(pt), -float(pt));
    sc.inv_p[t] = f2_pack(1.0f / float(pt), 1.0f / float(pt));
  }
  const int ndig = crt.q_bits + 1 <= 39 ? 3 : (crt.q_bits + 1 <= 58 ? 4 : 5);
  const long long base = ndig == 4 ? 32768 : 8192;
  for (int t = 0; t < L.nmod; ++t) {
    const int pt = crt.p[t];
    long long w = 1;
    for (int i = 0; i < 4; ++i) {
      w = (w * base) % pt;  // base^(i+1) mod p
      const float c = float(w > pt / 2 ? w - pt : w);
      sc.c[t][i] = f2_pack(c, c);
    }
  }
  *ndig_out = ndig;
  return sc;
}

// Residues of moduli t0 .. t1-1 of A (which & 1) and B (which & 2).
template <typename TIn>
void slice_operands(const oz::Layout& L, const oz::Crt& crt, const GemmProblem& p, bool cplx,
                    const int* sigA, const int* sigB, int8_t* resA, int8_t* resB, int t0, int t1,
                    int which, cudaStream_t st, int* status, double* ssqA = nullptr,
                    double* ssqB = nullptr) {
  using namespace oz;
  const TIn* A = static_cast<const TIn*>(p.A);
  const TIn* B = static_cast<const TIn*>(p.B);
  const int64_t ldA = cplx ? 2 * p.lda : p.lda;  // in real elements
  const int64_t ldB = cplx ? 2 * p.ldb : p.ldb;
  if (std::is_same<TIn, double>::value && cplx && t0 == 0 && t1 == L.nmod && crt.p[0] == 256 &&
      L.nmod >= 2 && !((which & 1) && L.mn) && !((which & 2) && L.mnB) && slice_tc_enabled()) {
    const double* Ad = reinterpret_cast<const double*>(A);
    const double* Bd = reinterpret_cast<const double*>(B);
    const bool okA = reinterpret_cast<uintptr_t>(Ad) % 16 == 0;
    const bool okB = reinterpret_cast<uintptr_t>(Bd) % 16 == 0;
    if ((!(which & 1) || okA) && (!(which & 2) || okB)) {
      const int64_t planeA = int64_t(L.rowsA) * L.kp, planeB = int64_t(L.nb) * L.kp;
      if (which & 1)
        launch_slice_tc(Ad, ldA, p.k, L.rowsA, L.kp, sigA, p.opA == 2 ? -1 : 1, resA,
                        int64_t(L.nsub) * planeA, planeA, crt, L.nmod, status, st);
      if (which & 2)
        launch_slice_tc(Bd, ldB, p.k, L.rowsB, L.kp, sigB, 1, resB, int64_t(L.nsub) * planeB,
                        planeB, crt, L.nmod, status, st);
      return;
    }
  }
  int ndig = 0;
  const SliceConsts sc = slice_consts(L, crt, &ndig);
  const int vec_elems = 16 / int(sizeof(TIn));
  const bool vecA = (reinterpret_cast<uintptr_t>(A) % 16 == 0) && (ldA % vec_elems == 0);
  const bool vecB = (reinterpret_cast<uintptr_t>(B) % 16 == 0) && (ldB % vec_elems == 0);
  // complex: three planes per modulus, A's third is re(a) - im(a) for A^H
  // (conj(a) b: Im = r2 - r0 + r1) and re(a) + im(a) otherwise; B's is re + im
  const int mode = cplx ? 2 : 0;
  const int sumA = p.opA == 2 ? -1 : 1;
  const int64_t strideA = int64_t(L.nsub) * L.rowsA * L.kp;
  const int64_t strideB = int64_t(L.nsub) * L.nb * L.kp;
  if ((which & 1) && L.mn)
    launch_slice_mn<TIn>(ndig, st, A, p.lda, L.rowsA, p.k, L.kp, sigA, mode, sumA, 0, resA,
                         strideA, sc, t0, t1);
  else if ((which & 1) && vecA)
    launch_slice<TIn, true>(ndig, st, A, ldA, L.K2, L.rowsA, L.kp, sigA, mode, sumA, resA,
                            strideA, sc, t0, t1, ssqA);
  else if (which & 1)
    launch_slice<TIn, false>(ndig, st, A, ldA, L.K2, L.rowsA, L.kp, sigA, mode, sumA, resA,
                             strideA, sc, t0, t1, ssqA);
  if ((which & 2) && L.mnB)  // op(B) = T or C: n-major rows, conjugated for C
    launch_slice_mn<TIn>(ndig, st, B, p.ldb, L.rowsB, p.k, L.kp, sigB, mode, 1,
                         p.opB == 2 ? 1 : 0, resB, strideB, sc, t0, t1);
  else if ((which & 2) && vecB)
    launch_slice<TIn, true>(ndig, st, B, ldB, L.K2, L.rowsB, L.kp, sigB, mode, 1, resB, strideB,
                            sc, t0, t1, ssqB);
  else if (which & 2)
    launch_slice<TIn, false>(ndig, st, B, ldB, L.K2, L.rowsB, L.kp, sigB, mode, 1, resB, strideB,
                             sc, t0, t1, ssqB);
}

// One-pass row scaling. The two-pass order reads every row twice: once for
// its norm (the scale exponent), once to slice it. Here the exponent comes
// from a sample of each row (16 evenly spread runs, 1/16 of its reals, the
// sum of squares extrapolated to the whole row) unless the estimated norm
// lies within kEstimateBand of a power of two, or the sample is zero or not
// finite: such rows (all of them for rows normalised to 1) take the exact
// norm at once. The default slicer also sums the squares of the scaled
// values, and an estimated exponent stands when that sum lies in
// [2^(2Q-2), 2^(2Q)) with a relative margin of 2^-30 at both ends (far above
// the rounding of either sum; see onepass_fixup): the scaled norm then lies in
// [2^(Q-1), 2^Q),
// which is what the exact exponent gives. Other rows (a sample that
// misjudged the row by more than the band) get the exact norm and are
// sliced again. Each row thus ends with the exponent and residues of the
// two-pass order, whatever the order of the atomic sums. Used for each
// k-major operand (an operand read in place keeps its norms) with the
// default modulus count and unrolled slicer, one modulus group and rows of
// at least kOnePassMinLen reals; SPLAB_OZAKI_ONEPASS=0 (read per call) keeps
// the two-pass order.
constexpr int64_t kOnePassMinLen = 131072;
constexpr int kOnePassRuns = 16;

// The operands scaled in one pass: bit 1 A, bit 2 B (k-major ones only; the
// rows read in place keep their k-sliced norms)
int onepass_operands(const oz::Layout& L, const GemmProblem& p, int groups) {
  const char* v = std::getenv("SPLAB_OZAKI_ONEPASS");
  if (v && v[0] == '0') return 0;
  const int nu = dtype_is_double(p.dtype) ? oz::kDefaultModuli : oz::kDefaultModuliFloat;
  if (!(p.k > 0 && groups == 1 && L.nmod == nu && slice_unroll() && !slice_tc_enabled() &&
        L.K2 >= kOnePassMinLen))
    return 0;
  return (L.mn ? 0 : 1) | (L.mnB ? 0 : 2);
}

// Exponents of A's (which & 1) and B's (which & 2) rows, estimated from the
// sample where that is safe, else exact (exact[row] = 1; p reads A k-major)
template <typename TIn>
void onepass_estimate(const oz::Layout& L, const oz::Crt& crt, const GemmProblem& p, bool cplx,
                      int* sigA, int* sigB, int* exactA, int* exactB, int which,
                      cudaStream_t st) {
  const int64_t run = (L.K2 / (16 * kOnePassRuns) + 7) / 8 * 8;  // reals per run
  const int64_t gap = L.K2 / kOnePassRuns;                         // run starts
  const int64_t ldA = cplx ? 2 * p.lda : p.lda, ldB = cplx ? 2 * p.ldb : p.ldb;
  if (which & 1)
    oz::oz_row_scale<TIn><<<L.rowsA, 256, 0, st>>>(static_cast<const TIn*>(p.A), ldA, L.K2,
                                                   L.rowsA, crt.q_bits, sigA, nullptr, nullptr,
                                                   kOnePassRuns, run, gap, exactA);
  if (which & 2)
    oz::oz_row_scale<TIn><<<L.rowsB, 256, 0, st>>>(static_cast<const TIn*>(p.B), ldB, L.K2,
                                                   L.rowsB, crt.q_bits, sigB, nullptr, nullptr,
                                                   kOnePassRuns, run, gap, exactB);
}

template <typename TIn, bool VEC, int EL, int MODE>
void launch_slice_rows_el(cudaStream_t st, const TIn* X, int64_t ld, int64_t len, int rows,
                          int64_t kp, const int* sig, int s_sign, int8_t* res, int64_t stride,
                          const oz::SliceConsts& sc, const int* list, const int* count) {
  using namespace oz;
  constexpr int kNU = sizeof(TIn) == 8 ? kDefaultModuli : kDefaultModuliFloat;
  constexpr int kDigU = sizeof(TIn) == 8 ? 4 : 3;
  const unsigned grid = unsigned((EL == 8 ? 4 : 2) * sm_count());  // one resident wave
  oz_slice_rows<TIn, VEC, kDigU, EL, kNU, MODE>
      <<<grid, 256, 0, st>>>(X, ld, len, rows, kp, sig, s_sign, res, stride, sc, list, count);
}

// The listed rows of one operand: exact exponent, then residues again
template <typename TIn>
void onepass_redo(const oz::Layout& L, const oz::Crt& crt, const oz::SliceConsts& sc,
                  const TIn* X, int64_t ld, int rows, int* sig, int s_sign, int8_t* res,
                  int64_t stride, int mode, const int* list, const int* count, cudaStream_t st) {
  oz::oz_row_scale<TIn><<<unsigned(std::min(rows, 2 * oz::sm_count())), 256, 0, st>>>(
      X, ld, L.K2, rows, crt.q_bits, sig, list, count);
  const bool vec = reinterpret_cast<uintptr_t>(X) % 16 == 0 && ld % (16 / int(sizeof(TIn))) == 0;
  auto run = [&](auto vec_tag, auto el_tag, auto mode_tag) {
    launch_slice_rows_el<TIn, decltype(vec_tag)::value, decltype(el_tag)::value,
                         decltype(mode_tag)::value>(st, X, ld, L.K2, rows, L.kp, sig, s_sign,
                                                    res, stride, sc, list, count);
  };
  using T = std::true_type;
  using F = std::false_type;
  using E8 = std::integral_constant<int, 8>;
  using E16 = std::integral_constant<int, 16>;
  using M0 = std::integral_constant<int, 0>;
  using M2 = std::integral_constant<int, 2>;
  const bool e16 = slice_elems() == 16;
  if (vec) {
    if (e16) mode == 2 ? run(T{}, E16{}, M2{}) : run(T{}, E16{}, M0{});
    else mode == 2 ? run(T{}, E8{}, M2{}) : run(T{}, E8{}, M0{});
  } else {
    if (e16) mode == 2 ? run(F{}, E16{}, M2{}) : run(F{}, E16{}, M0{});
    else mode == 2 ? run(F{}, E8{}, M2{}) : run(F{}, E8{}, M0{});
  }
}

// Check of A's (which & 1) and B's (which & 2) rows after slicing with their
// sums of squares, and the second pass over the rows it lists
template <typename TIn>
void onepass_fixup(const oz::Layout& L, const oz::Crt& crt, const GemmProblem& p, bool cplx,
                   int* sigA, int* sigB, int8_t* resA, int8_t* resB, double* ssq, int* list,
                   int which, cudaStream_t st) {
  using namespace oz;
  // the two sums of squares (norm kernel: runs of K2 / 256 terms per thread,
  // then trees; slicer: 8 terms per thread, trees, K2 / 2048 atomics per
  // row) differ by at most about (K2 / 256 + K2 / 2048 + 64) units of 2^-53
  // relative; the margin is 2^-30, or K2 2^-59 for rows beyond 2^29 reals
  const double delta = std::max(std::ldexp(1.0, -30), std::ldexp(double(L.K2), -59));
  const double lo = std::ldexp(1.0 + delta, 2 * crt.q_bits - 2);
  const double hi = std::ldexp(1.0 - delta, 2 * crt.q_bits);
  int* listA = list;
  int* listB = list + L.rowsA;
  const int* exactA = list + L.rowsA + L.rowsB;
  const int* exactB = exactA + L.rowsA;
  int* cnt = list + 2 * (L.rowsA + L.rowsB);  // A's count, B's count
  if (which & 1)
    oz_onepass_check<<<unsigned((L.rowsA + 255) / 256), 256, 0, st>>>(ssq, exactA, L.rowsA, lo,
                                                                     hi, listA, cnt);
  if (which & 2)
    oz_onepass_check<<<unsigned((L.rowsB + 255) / 256), 256, 0, st>>>(
        ssq + L.rowsA, exactB, L.rowsB, lo, hi, listB, cnt + 1);
  int ndig = 0;
  const SliceConsts sc = slice_consts(L, crt, &ndig);
  const int mode = cplx ? 2 : 0;
  const int64_t ldA = cplx ? 2 * p.lda : p.lda, ldB = cplx ? 2 * p.ldb : p.ldb;
  if (which & 1)
    onepass_redo<TIn>(L, crt, sc, static_cast<const TIn*>(p.A), ldA, L.rowsA, sigA,
                      p.opA == 2 ? -1 : 1, resA, int64_t(L.nsub) * L.rowsA * L.kp, mode, listA,
                      cnt, st);
  if (which & 2)
    onepass_redo<TIn>(L, crt, sc, static_cast<const TIn*>(p.B), ldB, L.rowsB, sigB, 1, resB,
                      int64_t(L.nsub) * L.nb * L.kp, mode, listB, cnt + 1, st);
}

// Side streams may be used by this host thread (off while a batch captures
// its sequence of contractions into a CUDA graph on one stream).
thread_local bool t_side_streams = true;

// Side streams of the modulus-group pipeline (per device): residues of group
// g + 1 are produced on `lo` while the GEMM of group g runs on `hi` (highest
// priority, so that its persistent CTAs are placed first and the slicing
// blocks fill the registers and issue slots the GEMM leaves free).
struct PipeStreams {
  cudaStream_t hi = nullptr, lo = nullptr;
  cudaEvent_t ev_start = nullptr, ev_done = nullptr, ev_scaled = nullptr,
              ev_sliced[oz::kMaxModuli] = {};
  std::mutex mu;  // one enqueue sequence at a time
  bool ok = false;
};

PipeStreams* pipe_streams() {
  static PipeStreams per_dev[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  PipeStreams& ps = per_dev[dev];
  static std::mutex init_mu;
  std::lock_guard<std::mutex> lk(init_mu);
  if (!ps.ok) {
    int lo_prio = 0, hi_prio = 0;
    bool good = cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio) == cudaSuccess &&
                cudaStreamCreateWithPriority(&ps.hi, cudaStreamNonBlocking, hi_prio) ==
                    cudaSuccess &&
                cudaStreamCreateWithPriority(&ps.lo, cudaStreamNonBlocking, lo_prio) ==
                    cudaSuccess &&
                cudaEventCreateWithFlags(&ps.ev_start, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&ps.ev_done, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&ps.ev_scaled, cudaEventDisableTiming) == cudaSuccess;
    for (int g = 0; good && g < oz::kMaxModuli; ++g)
      good = cudaEventCreateWithFlags(&ps.ev_sliced[g], cudaEventDisableTiming) == cudaSuccess;
    if (!good) {
      cudaGetLastError();
      return nullptr;
    }
    ps.ok = true;
  }
  return &ps;
}

// Number of modulus groups. Default 1: overlapping the slicing of one group
// with the GEMM of the previous one measured slower on B200 (both phases
// draw on L2 bandwidth; the slicing ran at half speed beside the GEMM).
// SPLAB_OZAKI_GROUPS = 2 .. number of moduli enables the pipeline.
int modulus_groups(const oz::Layout& L) {
  int g = 1;
  if (const char* v = std::getenv("SPLAB_OZAKI_GROUPS")) {
    const int f = std::atoi(v);
    if (f > 0) g = f;
  }
  return std::max(1, std::min(g, L.nmod));
}
}  // namespace

namespace {
// Tensor-core CRT reconstruction (oz_reconstruct_tc), the default for byte
// residues (one k-chunk) with m % 16 == 0, m >= 128 and at most 64 product
// planes; SPLAB_OZAKI_RECON_TC=0 (read per call) selects the CUDA-core
// kernels. True when it applies and its tensor map was made.
bool recon_tc_plan(const oz::Layout& L, unsigned char* R8, CUtensorMap* map) {
  using namespace oz;
  const char* v = std::getenv("SPLAB_OZAKI_RECON_TC");
  if ((v && v[0] == '0') || !R8 || L.nmod * L.nsub > RT_KP || L.rowsA % 16 != 0 ||
      L.rowsA < 128)
    return false;
  return make_map_recon(map, R8, L.rowsA, L.nb, L.nmod * L.nsub);
}

cudaError_t launch_recon_tc(const GemmProblem& p, const oz::Layout& L, const oz::Crt& crt,
                            const oz::ReconParams& rp, const CUtensorMap& map, const int* sigA,
                            const int* sigB, int* status, cudaStream_t st) {
  using namespace oz;
  const bool cplx = dtype_is_complex(p.dtype);
  const int planes = L.nmod * L.nsub;
  static thread_local ReconTcParams P;  // 2.7 KB: kept off the stack
  P = ReconTcParams{};
  P.m = L.rowsA;
  P.n = int(p.n);
  P.row_blocks = (P.m + 128 * RT_G - 1) / (128 * RT_G);
  P.total_units = (long long)P.row_blocks * P.n;
  P.planes = planes;
  P.kp = planes <= 32 ? 32 : 64;
  P.sigA = sigA;
  P.sigB = sigB;
  P.C = p.C;
  P.ldc = p.ldc;
  P.alr = p.alpha[0];
  P.ali = p.alpha[1];
  P.ber = p.beta[0];
  P.bei = p.beta[1];
  P.fill = p.fill_mode;
  P.ro = p.fill_ro;
  P.co = p.fill_co;
  P.tile_m = BM;
  P.tile_n = cplx ? BN / 2 : BN;
  P.rp = rp;
  // weight bytes: plane k = t * nsub + s takes W_t or P - W_t (the combination
  // of combine3 with its signs carried by the weights)
  const unsigned __int128 Pm = (unsigned __int128)crt.P_hi << 64 | crt.P_lo;
  for (int t = 0; t < L.nmod; ++t) {
    const unsigned __int128 W = (unsigned __int128)crt.w_hi[t] << 64 | crt.w_lo[t];
    const unsigned __int128 Wn = Pm - W;
    for (int s = 0; s < L.nsub; ++s) {
      unsigned __int128 vre = W, vim = 0;
      if (cplx) {
        if (s == 0) {
          vre = W;
          vim = Wn;
        } else if (s == 1) {
          vre = rp.conj ? W : Wn;
          vim = rp.conj ? W : Wn;
        } else {
          vre = 0;
          vim = W;
        }
      }
      const int k = t * L.nsub + s;
      for (int o = 0; o < 16; ++o) {
        P.v[o][k] = static_cast<unsigned char>(vre >> (8 * o));
        P.v[16 + o][k] = static_cast<unsigned char>(vim >> (8 * o));
      }
    }
  }
  P.status = status;
  P.wait_limit_ns = kWaitLimitNs;
  auto run = [&](auto kern) -> cudaError_t {
    const cudaError_t ea = set_dynamic_smem(reinterpret_cast<const void*>(kern), RT_SMEM);
    if (ea != cudaSuccess) return ea;
    // three CTAs per SM (their shared memory fits, and so their TMEM)
    const long long grid = std::min<long long>(P.total_units, 3LL * sm_count());
    kern<<<unsigned(grid), RT_THREADS, RT_SMEM, st>>>(map, P);
    return cudaGetLastError();
  };
  switch (p.dtype) {
    case kC64: return run(oz_reconstruct_tc<kC64>);
    case kC32: return run(oz_reconstruct_tc<kC32>);
    case kR64: return run(oz_reconstruct_tc<kR64>);
    default: return run(oz_reconstruct_tc<kR32>);
  }
}

// At <- A k-major (op(A) = N operands); see oz_transpose
cudaError_t transpose_a(const GemmProblem& p, const oz::Layout& L, void* At, cudaStream_t st) {
  const dim3 block(32, 8);
  const dim3 grid(unsigned((p.m + 31) / 32),
                  unsigned(std::min<int64_t>((p.k + 31) / 32, 65535)));
  auto run = [&](auto tag) {
    using E = decltype(tag);
    oz::oz_transpose<E><<<grid, block, 0, st>>>(static_cast<const E*>(p.A), p.lda, int(p.m),
                                                p.k, static_cast<E*>(At), L.ldAt);
  };
  switch (p.dtype) {
    case kC64: run(double2{}); break;
    case kC32: run(float2{}); break;
    case kR64: run(double{}); break;
    default: run(float{}); break;
  }
  return cudaGetLastError();
}
}  // namespace

cudaError_t ozaki_gemm(const GemmProblem& p_in, int moduli, void* ws, size_t ws_bytes,
                       cudaStream_t st) {
  using namespace oz;
  if (!ozaki_supported(p_in)) return cudaErrorNotSupported;
  if (p_in.m <= 0 || p_in.n <= 0) return cudaSuccess;
  const Layout L = layout_of(p_in, moduli);
  if (ws_bytes < L.total || !ws) return cudaErrorInvalidValue;
  const Crt crt = make_crt(L.nmod);
  const bool cplx = dtype_is_complex(p_in.dtype);
  char* w = static_cast<char*>(ws);
  int* sigA = reinterpret_cast<int*>(w + L.off_sigA);
  int* sigB = reinterpret_cast<int*>(w + L.off_sigB);
  int8_t* resA = reinterpret_cast<int8_t*>(w + L.off_resA);
  int8_t* resB = reinterpret_cast<int8_t*>(w + L.off_resB);
  int* R = reinterpret_cast<int*>(w + L.off_R);
  unsigned char* R8 = L.r8 ? reinterpret_cast<unsigned char*>(w + L.off_R) : nullptr;
  int* status = reinterpret_cast<int*>(w + L.off_status);
  // byte residues of C, where they apply, go to the tensor-core reconstruction
  CUtensorMap rmap;
  const bool tc_recon = p_in.k > 0 && recon_tc_plan(L, R8, &rmap);

  cudaError_t e;
  // op(A) = N: everything below reads the k-major copy At as op(A) = T
  GemmProblem p = p_in;
  if (L.at && p.k > 0) {
    p.A = w + L.off_At;
    p.lda = L.ldAt;
    p.opA = 1;
  }
  const bool dbl = dtype_is_double(p.dtype);
  const int groups = modulus_groups(L);
  // Large problems use the side streams: the row norms of B (a pure read)
  // run beside the slicing of A (arithmetic-bound), and with groups > 1 the
  // modulus-group pipeline below.
  const bool big = double(L.rowsA + L.rowsB) * double(L.K2) * dtype_bytes(p.dtype) /
                       (cplx ? 2.0 : 1.0) >= 5e8;
  static const bool side_norms = [] {
    const char* v = std::getenv("SPLAB_OZAKI_SIDE_NORMS");
    return !(v && v[0] == '0');
  }();
  const int onepass = onepass_operands(L, p, groups);
  double* ssq = reinterpret_cast<double*>(w + L.off_ssq);
  int* oplist = reinterpret_cast<int*>(w + L.off_list);
  PipeStreams* ps =
      (p.k > 0 && (groups > 1 || (big && side_norms)) && t_side_streams)
          ? pipe_streams()
          : nullptr;
  std::unique_lock<std::mutex> lk;
  if (ps) lk = std::unique_lock<std::mutex>(ps->mu);
  auto scale = [&](int which, cudaStream_t s) {
    if (dbl)
      scale_operands<double>(L, crt, p, cplx, sigA, sigB, w, which, s);
    else
      scale_operands<float>(L, crt, p, cplx, sigA, sigB, w, which, s);
  };
  phase_mark(0, false, st);
  if (L.at && p.k > 0) {
    phase_mark(15, false, st);
    if ((e = transpose_a(p_in, L, w + L.off_At, st)) != cudaSuccess) return e;
    phase_mark(15, true, st);
  }
  // row exponents of A (which & 1) and B (which & 2): estimated for the
  // operands scaled in one pass, else the exact norms
  int* exactA = oplist + L.rowsA + L.rowsB;
  auto exponents = [&](int which, cudaStream_t s) {
    if (which & onepass) {
      if (dbl)
        onepass_estimate<double>(L, crt, p, cplx, sigA, sigB, exactA, exactA + L.rowsA,
                                 which & onepass, s);
      else
        onepass_estimate<float>(L, crt, p, cplx, sigA, sigB, exactA, exactA + L.rowsA,
                                which & onepass, s);
    }
    if (which & ~onepass) scale(which & ~onepass, s);
  };
  if (onepass && ((e = cudaMemsetAsync(ssq, 0, sizeof(double) * (size_t(L.rowsA) + L.rowsB),
                                       st)) != cudaSuccess ||
                  (e = cudaMemsetAsync(oplist + 2 * (L.rowsA + L.rowsB), 0, 2 * sizeof(int),
                                       st)) != cudaSuccess))
    return e;
  const bool side_exponents = p.k > 0 && ps && onepass != 1;
  if (side_exponents) {
    // A's exponents alone (norms are pure reads and would share the
    // bandwidth), then B's on the side stream while A is sliced
    phase_mark(16, false, st);
    exponents(1, st);
    phase_mark(16, true, st);
    if ((e = cudaEventRecord(ps->ev_start, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ps->lo, ps->ev_start, 0)) != cudaSuccess) return e;
    exponents(2, ps->lo);
    if ((e = cudaEventRecord(ps->ev_scaled, ps->lo)) != cudaSuccess) return e;
  } else if (p.k > 0) {
    // B's exact norms first, alone, when only A is scaled in one pass: beside
    // A's slicing with its sums of squares they measured slower (op(A) = C,
    // op(B) = C at the headline size: 18.2 against 18.0 ms for two passes)
    phase_mark(16, false, st);
    exponents(2, st);
    exponents(1, st);
    phase_mark(16, true, st);
  } else {
    cudaMemsetAsync(sigA, 0, sizeof(int) * L.rowsA, st);
    cudaMemsetAsync(sigB, 0, sizeof(int) * L.rowsB, st);
  }
  // byte residues are stored, not accumulated: every element the
  // reconstruction reads is written by the GEMM
  if (!L.r8)
    cudaMemsetAsync(R, 0, sizeof(int) * size_t(L.nmod) * L.nsub * L.nb * L.rowsA, st);
  cudaMemsetAsync(status, 0, sizeof(int), st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (p.k <= 0) {
    phase_mark(0, true, st);
    phase_mark(1, false, st);
    phase_mark(1, true, st);
  } else {
    // with one-pass scaling the slicer also sums the rows' scaled squares
    double* ssqA = (onepass & 1) ? ssq : nullptr;
    double* ssqB = (onepass & 2) ? ssq + L.rowsA : nullptr;
    auto slice = [&](int t0, int t1, int which, cudaStream_t s) {
      if (dbl)
        slice_operands<double>(L, crt, p, cplx, sigA, sigB, resA, resB, t0, t1, which, s,
                               status, ssqA, ssqB);
      else
        slice_operands<float>(L, crt, p, cplx, sigA, sigB, resA, resB, t0, t1, which, s,
                              status, ssqA, ssqB);
    };
    CUtensorMap mapA, mapB;
    if (!make_map(&mapA, resA, L.kp, int64_t(L.nmod) * L.nsub * L.rowsA, BM) ||
        !make_map(&mapB, resB, L.kp, int64_t(L.nmod) * L.nsub * L.nb, BN))
      return cudaErrorNotSupported;
    GemmParams g{};
    g.m = L.rowsA;
    g.nb = L.nb;
    g.kblocks = int(L.kp / BKB);
    g.nchunks = (g.kblocks + kChunkBlocks - 1) / kChunkBlocks;
    // equal chunks (each within the exact INT32 bound): equal work units
    g.chunk_blocks = std::max(1, (g.kblocks + g.nchunks - 1) / std::max(1, g.nchunks));
    g.nmod = L.nmod * L.nsub;
    g.nsub = L.nsub;
    g.tiles_m = (L.rowsA + BM - 1) / BM;
    g.tiles_n = (L.nb + BN - 1) / BN;
    g.total_units = g.nmod * g.nchunks * g.tiles_m * g.tiles_n;
    g.R = R;
    g.R8 = R8;
    g.status = status;
    g.wait_limit_ns = kWaitLimitNs;
    g.stall_test = 0;
    if (const char* v = std::getenv("SPLAB_OZAKI_STALL_TEST")) {
      // test hook for the failure path: no copies are issued, every wait runs
      // into a 50 ms bound, the kernel reports SPLAB_ERR_TIMEOUT and returns
      if (v[0] == '1') {
        g.stall_test = 1;
        g.wait_limit_ns = 50000000ull;
      }
    }
    // short units (few k-blocks): two epilogue warps per lane quarter
    g.epi_split = g.chunk_blocks < 128 ? 2 : 1;
    if (const char* v = std::getenv("SPLAB_OZAKI_EPI_SPLIT")) {
      if (v[0] == '1') g.epi_split = 1;
      if (v[0] == '2') g.epi_split = 2;
    }
    for (int t = 0; t < L.nmod; ++t) {
      g.p[t] = crt.p[t];
      const ModMagic mm = make_mod_magic(crt.p[t]);
      g.c16[t] = mm.c16;
      g.off[t] = mm.off;
      g.M[t] = mm.M;
    }
    const char* gk = std::getenv("SPLAB_OZAKI_GEMM");
    const bool pair = !(gk && gk[0] == '1');  // "1sm" selects the single-CTA kernel
    CUtensorMap mapA2, mapB2;
    // pair tile 256 x 512 (one A tile for two MMAs, one 512-column
    // accumulator drained once per unit) when the units are long enough to
    // hide the drain (128 k-blocks or more) and it needs at most 5 % more
    // rounds of work units than the double-buffered 256 x 256 tile; measured
    // 9 % faster on the INT8 GEMM of m = n = 1024, k = 250000 (complex double
    // and float) under the power cap (SPLAB_OZAKI_NT=1|2 overrides)
    int nt = 1;
    if (L.nb >= 512 && g.chunk_blocks >= 128) {
      const int pairs = std::max(1, sm_count() / 2);
      auto rounds = [&](int w) {
        const long long units = (long long)g.nmod * g.nchunks * ((L.rowsA + 255) / 256) *
                                ((L.nb + 256 * w - 1) / (256 * w));
        return double((units + pairs - 1) / pairs);
      };
      nt = rounds(2) * 2.0 <= rounds(1) * 1.05 ? 2 : 1;
    }
    if (const char* v = std::getenv("SPLAB_OZAKI_NT")) {
      if (v[0] == '1') nt = 1;
      if (v[0] == '2') nt = 2;
    }
    const int tile_nb = 256 * nt;
    if (pair) {
      g.tiles_m = (L.rowsA + 255) / 256;
      g.tiles_n = (L.nb + tile_nb - 1) / tile_nb;
      g.total_units = g.nmod * g.nchunks * g.tiles_m * g.tiles_n;
      if (p.fill_mode != 0) {
        // compute only the pair tiles that cover an element the reconstruction
        // writes: its tiles are BM x (BN/2 complex | BN real) of C; a pair tile
        // covers rows r0 .. r1-1 and columns b0 .. b1-1 of C (B rows = columns)
        const int rt_m = BM, rt_n = cplx ? BN / 2 : BN;
        std::vector<int> act;
        for (int tn = 0; tn < g.tiles_n; ++tn)
          for (int tm = 0; tm < g.tiles_m; ++tm) {
            const int64_t r0 = int64_t(tm) * 256, r1 = std::min<int64_t>(r0 + 256, L.rowsA);
            const int64_t b0 = int64_t(tn) * tile_nb, b1 = std::min<int64_t>(b0 + tile_nb, L.nb);
            bool on = false;
            for (int64_t ti = (r0 / rt_m) * rt_m; ti < r1 && !on; ti += rt_m)
              for (int64_t tj = (b0 / rt_n) * rt_n; tj < b1 && !on; tj += rt_n)
                on = tile_is_active(p.fill_mode, ti, tj, std::min<int64_t>(rt_m, p.m - ti),
                                    std::min<int64_t>(rt_n, p.n - tj), p.fill_ro, p.fill_co);
            if (on) act.push_back(tm + tn * g.tiles_m);
          }
        if (act.empty()) act.push_back(0);  // keep the launch well formed
        int* dtiles = reinterpret_cast<int*>(w + L.off_tiles);
        if ((e = cudaMemcpyAsync(dtiles, act.data(), sizeof(int) * act.size(),
                                 cudaMemcpyHostToDevice, st)) != cudaSuccess)
          return e;
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;  // host list goes away
        g.active = dtiles;
        g.n_active = int(act.size());
        g.total_units = g.nmod * g.nchunks * g.n_active;
      }
      if ((e = set_dynamic_smem(reinterpret_cast<const void*>(oz_gemm_pair<1>),
                                PairCfg<1>::SMEM)) != cudaSuccess ||
          (e = set_dynamic_smem(reinterpret_cast<const void*>(oz_gemm_pair<2>),
                                PairCfg<2>::SMEM)) != cudaSuccess)
        return e;
      if (!make_map(&mapA2, resA, L.kp, int64_t(L.nmod) * L.nsub * L.rowsA, 128) ||
          !make_map(&mapB2, resB, L.kp, int64_t(L.nmod) * L.nsub * L.nb, 128))
        return cudaErrorNotSupported;
    }
    const int units_per_mod = g.total_units / L.nmod;  // all products of one modulus
    // the INT8 GEMM over moduli t0 .. t1-1 on stream s
    auto launch_gemm = [&](int t0, int t1, cudaStream_t s) -> cudaError_t {
      GemmParams gg = g;
      gg.t0 = t0 * L.nsub;
      gg.total_units = (t1 - t0) * units_per_mod;
      if (pair) {
        const int pairs = std::max(1, std::min(gg.total_units, sm_count() / 2));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(unsigned(2 * pairs));
        cfg.blockDim = dim3(PAIR_THREADS);
        cfg.dynamicSmemBytes = nt == 2 ? PairCfg<2>::SMEM : PairCfg<1>::SMEM;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 2;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return nt == 2 ? cudaLaunchKernelEx(&cfg, oz_gemm_pair<2>, mapA2, mapB2, gg)
                       : cudaLaunchKernelEx(&cfg, oz_gemm_pair<1>, mapA2, mapB2, gg);
      }
      const cudaError_t ea = set_dynamic_smem(reinterpret_cast<const void*>(oz_gemm), GEMM_SMEM);
      if (ea != cudaSuccess) return ea;
      const int grid = std::min(gg.total_units, sm_count());
      oz_gemm<<<grid, GEMM_THREADS, GEMM_SMEM, s>>>(mapA, mapB, gg);
      return cudaGetLastError();
    };

    if (groups == 1 || !ps) {
      phase_mark(17, false, st);
      slice(0, L.nmod, 1, st);  // A on the caller's stream
      phase_mark(17, true, st);
      // B once its row norms are done (on the side stream when there is one)
      if (side_exponents && (e = cudaStreamWaitEvent(st, ps->ev_scaled, 0)) != cudaSuccess)
        return e;
      phase_mark(18, false, st);
      slice(0, L.nmod, 2, st);
      phase_mark(18, true, st);
      if (onepass) {
        phase_mark(19, false, st);
        if (dbl)
          onepass_fixup<double>(L, crt, p, cplx, sigA, sigB, resA, resB, ssq, oplist, onepass,
                                st);
        else
          onepass_fixup<float>(L, crt, p, cplx, sigA, sigB, resA, resB, ssq, oplist, onepass,
                               st);
        phase_mark(19, true, st);
      }
      phase_mark(0, true, st);
      phase_mark(1, false, st);
      phase_mark(3, false, st);
      if ((e = launch_gemm(0, L.nmod, st)) != cudaSuccess) return e;
      phase_mark(3, true, st);
      phase_mark(1, true, st);
    } else {
      // modulus-group pipeline: slicing of group i + 1 (stream lo) overlaps
      // the GEMM of group i (stream hi); the caller's stream joins at the end
      auto bounds = [&](int i) { return i * L.nmod / groups; };
      // lo has the B row norms queued; it also needs A's row norms and the
      // memsets of the caller's stream
      if ((e = cudaEventRecord(ps->ev_start, st)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(ps->lo, ps->ev_start, 0)) != cudaSuccess) return e;
      for (int i = 0; i < groups; ++i) {
        slice(bounds(i), bounds(i + 1), 3, ps->lo);
        if ((e = cudaEventRecord(ps->ev_sliced[i], ps->lo)) != cudaSuccess) return e;
      }
      phase_mark(0, true, ps->lo);
      for (int i = 0; i < groups; ++i) {
        if ((e = cudaStreamWaitEvent(ps->hi, ps->ev_sliced[i], 0)) != cudaSuccess) return e;
        if (i == 0) phase_mark(1, false, ps->hi);
        phase_mark(3 + i, false, ps->hi);
        if ((e = launch_gemm(bounds(i), bounds(i + 1), ps->hi)) != cudaSuccess) return e;
        phase_mark(3 + i, true, ps->hi);
      }
      phase_mark(1, true, ps->hi);
      if ((e = cudaEventRecord(ps->ev_done, ps->hi)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(st, ps->ev_done, 0)) != cudaSuccess) return e;
    }
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;

  phase_mark(2, false, st);
  ReconParams rp = make_recon(crt);
  rp.conj = p.opA == 2 ? 1 : 0;
  // threads along the rows of C, one block row covering all of them (no
  // partial second pass), blocks along the columns (grid-stride beyond
  // 65535); byte residues with m % 16 == 0 take the shared-memory staged
  // kernel instead
  const int threads = 256;
  const bool staged = R8 && L.rowsA % 16 == 0;
  const unsigned gy = unsigned(std::min<int64_t>(p.n, 65535));
  const unsigned gx = unsigned(std::max<int64_t>(1, (p.m + threads - 1) / threads));
  const bool fixed = L.nmod == (dtype_is_double(p.dtype) ? kDefaultModuli : kDefaultModuliFloat);
  if (tc_recon) {
    if ((e = launch_recon_tc(p, L, crt, rp, rmap, sigA, sigB, status, st)) != cudaSuccess)
      return e;
    phase_mark(2, true, st);
    return cudaGetLastError();
  }
  if (staged) {
    const int smem = staged_smem_bytes(cplx, L.nmod);
    const int64_t items = (p.m + kStageRows - 1) / kStageRows * p.n;
    const unsigned grid = unsigned(std::min<int64_t>(items, int64_t(2) * sm_count()));
    auto run = [&](auto kern) -> cudaError_t {
      const cudaError_t ea = set_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
      if (ea != cudaSuccess) return ea;
      kern<<<grid, threads, smem, st>>>(R8, L.rowsA, int(p.n), L.nb, sigA, sigB, p.C, p.ldc,
                                        p.alpha[0], p.alpha[1], p.beta[0], p.beta[1],
                                        p.fill_mode, p.fill_ro, p.fill_co, BM,
                                        cplx ? BN / 2 : BN, rp);
      return cudaGetLastError();
    };
    switch (p.dtype) {
      case kC64:
        e = fixed ? run(oz_reconstruct_staged<kC64, kDefaultModuli>)
                  : run(oz_reconstruct_staged<kC64, 0>);
        break;
      case kC32:
        e = fixed ? run(oz_reconstruct_staged<kC32, kDefaultModuliFloat>)
                  : run(oz_reconstruct_staged<kC32, 0>);
        break;
      case kR64:
        e = fixed ? run(oz_reconstruct_staged<kR64, kDefaultModuli>)
                  : run(oz_reconstruct_staged<kR64, 0>);
        break;
      default:
        e = fixed ? run(oz_reconstruct_staged<kR32, kDefaultModuliFloat>)
                  : run(oz_reconstruct_staged<kR32, 0>);
        break;
    }
    if (e != cudaSuccess) return e;
    phase_mark(2, true, st);
    return cudaGetLastError();
  }
  auto recon = [&](auto kern, const auto* Rsrc) {
    kern<<<dim3(gx, gy), threads, 0, st>>>(Rsrc, L.rowsA, int(p.n), L.nb, sigA, sigB, p.C, p.ldc,
                                           p.alpha[0], p.alpha[1], p.beta[0], p.beta[1],
                                           p.fill_mode, p.fill_ro, p.fill_co, BM,
                                           cplx ? BN / 2 : BN, rp);
  };
  using u8 = unsigned char;
  // the default modulus counts (15 double, 9 float) run a fully unrolled
  // reconstruction
  auto by_dtype = [&](auto rt_tag, const auto* Rsrc) {
    using RT = decltype(rt_tag);
    switch (p.dtype) {
      case kC64:
        fixed ? recon(oz_reconstruct<kC64, RT, kDefaultModuli>, Rsrc)
              : recon(oz_reconstruct<kC64, RT, 0>, Rsrc);
        break;
      case kC32:
        fixed ? recon(oz_reconstruct<kC32, RT, kDefaultModuliFloat>, Rsrc)
              : recon(oz_reconstruct<kC32, RT, 0>, Rsrc);
        break;
      case kR64:
        fixed ? recon(oz_reconstruct<kR64, RT, kDefaultModuli>, Rsrc)
              : recon(oz_reconstruct<kR64, RT, 0>, Rsrc);
        break;
      default:
        fixed ? recon(oz_reconstruct<kR32, RT, kDefaultModuliFloat>, Rsrc)
              : recon(oz_reconstruct<kR32, RT, 0>, Rsrc);
        break;
    }
  };
  if (R8)
    by_dtype(u8{}, R8);
  else
    by_dtype(int{}, R);
  phase_mark(2, true, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return cudaSuccess;
}

int* ozaki_status_ptr(const GemmProblem& p, int moduli, void* ws) {
  return reinterpret_cast<int*>(static_cast<char*>(ws) + oz::layout_of(p, moduli).off_status);
}

void ozaki_allow_side_streams(bool allow) { t_side_streams = allow; }

int ozaki_status(const GemmProblem& p, int moduli, void* ws, cudaStream_t st) {
  const oz::Layout L = oz::layout_of(p, moduli);
  int h = 0;
  cudaMemcpyAsync(&h, static_cast<char*>(ws) + L.off_status, sizeof(int), cudaMemcpyDeviceToHost,
                  st);
  cudaStreamSynchronize(st);
  return h;
}

}  // namespace splab
