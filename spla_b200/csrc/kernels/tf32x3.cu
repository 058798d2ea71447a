// 3xTF32 contraction for float and complex float on tcgen05 (sm_100a).
//
// C <- alpha * op(A) * B + beta * C with op(A) in {T, C} (the pgemm_ssb
// layout). Each float x is split into x_hi = tf32(x) and x_lo = tf32(x - x_hi)
// (both rounded to nearest), and the product is taken as
// a_hi b_hi + a_hi b_lo + a_lo b_hi on the TF32 tensor cores; the dropped
// a_lo b_lo term and the TF32 rounding of the low parts are ~2^-22 relative.
// Complex operands use the real form of the Ozaki path: rows of op(A) read as
// 2k reals against u_j = (br, -s bi) and v_j = (bi, s br).
//
// Accumulation precision. The tensor cores add into an FP32 accumulator with
// a truncating (biased) rounding, so an accumulation chain of L MMAs over
// sign-coherent terms (the diagonal of an overlap matrix A^H A) loses about
// L/2 units in the last place. Long FP32 chains are therefore avoided: k is
// walked in windows of kWin k-blocks (64 reals); each window starts from a
// zero accumulator, issues the small correction products (hi lo, lo hi) of
// the whole window first and the hi hi products last, so only 8 MMAs add
// into a large value. The epilogue adds kFold window results in registers
// (round to nearest), folds that sum into a running double-float sum (hi +
// lo pair of FP32, error-free 2Sum) kept in TMEM beside the double-buffered
// accumulator, and writes the FP64 value of the sum once per work unit.
//
// Tiles: a CTA pair computes 256 rows x 128 columns of the real-form result
// (tcgen05.mma.cta_group::2.kind::tf32 M256 N128 K8). TMEM per CTA: columns
// 0-255 two FP32 accumulators, 256-383 sum hi, 384-511 sum lo. A work unit
// is one tile over a super-chunk of k; the reduction kernel sums the FP64
// partials of the super-chunks in order, assembles complex values and
// applies alpha / beta.
//
// Kernels: tf3_split (hi/lo planes, K-major, u/v rows for complex B),
// tf3_gemm_pair (TMA -> smem ring -> tensor cores -> TMEM sums -> FP64
// partials), tf3_reduce.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "gemm_dmma.cuh"
#include "tcgen05_common.cuh"
#include "tf32x3.cuh"

namespace splab {
namespace tf3 {
using namespace tc;

constexpr int BKF = 32;                 // floats per k-block (one 128-byte swizzle atom)
constexpr int TN = 128;                 // tile columns (real-form rows of B) per CTA pair
constexpr int A_PLANE = 128 * 128;      // bytes per A plane per CTA and stage (128 rows)
constexpr int B_PLANE = 64 * 128;       // bytes per B plane per CTA and stage (64 rows)
constexpr int STAGE_BYTES = 2 * A_PLANE + 2 * B_PLANE;  // A_hi, A_lo, B_hi, B_lo
constexpr int STAGES = 4;
constexpr int kWin = 2;                 // k-blocks per FP32 accumulation window
constexpr int kFold = 4;                // windows per register sum before the 2Sum fold
constexpr int kMinSuperBlocks = 64;     // smallest k extent of a work unit (2048 reals)
constexpr int THREADS = 320;            // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr int SMEM = STAGES * STAGE_BYTES + 2048;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;
constexpr uint32_t kIdesc = (1u << 4)                      // D: F32
                            | (2u << 7) | (2u << 10)       // A, B: TF32
                            | (uint32_t(TN >> 3) << 17)    // N = 128
                            | (uint32_t(256 >> 4) << 24);  // M = 256 (CTA pair)
static_assert(STAGES >= 2 * kWin, "the ring holds the window being multiplied and the next one");

__device__ __forceinline__ float tf32_rn(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r & 0xFFFFE000u);
}

// hi/lo planes of one operand, K-major, row stride kp floats; each thread
// handles 4 consecutive reals of one row. mode 1: complex B -> u rows `row`,
// v rows `row + rows`.
__global__ void tf3_split(const float* __restrict__ X, int64_t ld, int64_t len, int rows,
                          int64_t kp, int mode, int s_sign, float* __restrict__ hi,
                          float* __restrict__ lo) {
  const int64_t groups = kp / 4;
  const int64_t gid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int row = int(gid / groups);
  if (row >= rows) return;
  const int64_t l0 = (gid % groups) * 4;
  const float* x = X + int64_t(row) * ld + l0;
  float v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = (l0 + i < len) ? x[i] : 0.0f;
  auto put = [&](int64_t r, const float (&w)[4]) {
    float h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      h[i] = tf32_rn(w[i]);
      l[i] = tf32_rn(w[i] - h[i]);
    }
    *reinterpret_cast<float4*>(hi + r * kp + l0) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(lo + r * kp + l0) = make_float4(l[0], l[1], l[2], l[3]);
  };
  if (mode == 0) {
    put(row, v);
  } else {
    const float s = float(s_sign);
    const float u[4] = {v[0], -s * v[1], v[2], -s * v[3]};
    const float w[4] = {v[1], s * v[0], v[3], s * v[2]};
    put(row, u);
    put(int64_t(row) + rows, w);
  }
}

struct GemmParams {
  int m, nb;          // rows of A and of B (real form)
  int kblocks;        // kp / 32
  int super_blocks;   // k-blocks per work unit
  int nsuper;         // super-chunks of k
  int tiles_m, tiles_n;
  int total_units;
  double* P;          // FP64 partials [nsuper][nb][m]
  int* status;
  const int* active;  // tiles to compute (fill mode) or null
  int n_active;
  unsigned long long wait_limit_ns;
  int stall_test;  // 1: the producer issues no copies (exercises the bounded waits)
};

__device__ __forceinline__ void umma_tf32_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
      : "memory");
}

// Error-free sum of two floats: a + b = t + e exactly (Knuth's 2Sum).
__device__ __forceinline__ void two_sum(float a, float b, float& t, float& e) {
  t = __fadd_rn(a, b);
  const float bp = __fsub_rn(t, a);
  const float ap = __fsub_rn(t, bp);
  e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
}

__global__ void __launch_bounds__(THREADS, 1)
    tf3_gemm_pair(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                  const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                  const __grid_constant__ GemmParams g) {
  extern __shared__ unsigned char smem_raw[];
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
  const uint32_t rank = cluster_rank();  // 0: issues the MMAs
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  const int tiles = g.tiles_m * g.tiles_n;
  const int ntl = g.active ? g.n_active : tiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);
      mbar_init(acce_bar(b), 16);  // one arrival per epilogue warp of both CTAs
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

  auto unit_of = [&](int u, int& sc, int& tm, int& tn) {
    const int tl = u % ntl;
    const int tile = g.active ? g.active[tl] : tl;
    tm = tile % g.tiles_m;
    tn = tile / g.tiles_m;
    sc = u / ntl;
  };

  bool aborted = false;
  if (warp == 0 && lane == 0) {
    // ---- TMA producer (both CTAs): 128 rows of A, 64 rows of B per plane
    int stage = 0;
    uint32_t phase = 0;
    bool ok = g.stall_test == 0;
    for (int u = pair; u < g.total_units && ok; u += npairs) {
      int sc, tm, tn;
      unit_of(u, sc, tm, tn);
      const int kb0 = sc * g.super_blocks, kb1 = min(g.kblocks, kb0 + g.super_blocks);
      const int arow = tm * 256 + int(rank) * 128;
      const int brow = tn * TN + int(rank) * (TN / 2);
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!mbar_wait(empty_bar(stage), phase ^ 1u, abort, g.wait_limit_ns)) {
          ok = false;
          break;
        }
        const uint32_t fb = map_to_rank(full_bar(stage), 0);
        if (rank == 0) mbar_arrive_expect_tx(full_bar(stage), 2 * STAGE_BYTES);
        const uint32_t sa = base + stage * STAGE_BYTES;
        tma_load_2d_pair(sa, &mAh, kb * BKF, arow, fb);
        tma_load_2d_pair(sa + A_PLANE, &mAl, kb * BKF, arow, fb);
        tma_load_2d_pair(sa + 2 * A_PLANE, &mBh, kb * BKF, brow, fb);
        tma_load_2d_pair(sa + 2 * A_PLANE + B_PLANE, &mBl, kb * BKF, brow, fb);
        if (++stage == STAGES) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
    aborted = !ok && g.stall_test == 0;
  } else if (warp == 1 && lane == 0 && rank == 0) {
    // ---- MMA issuer (even CTA): per window, corrections first, hi hi last
    int stage = 0;
    uint32_t phase = 0;
    uint32_t acc_phase[2] = {0, 0};
    int accb = 0;
    bool ok = true;
    for (int u = pair; u < g.total_units && ok; u += npairs) {
      int sc, tm, tn;
      unit_of(u, sc, tm, tn);
      const int kb0 = sc * g.super_blocks, kb1 = min(g.kblocks, kb0 + g.super_blocks);
      for (int w0 = kb0; w0 < kb1 && ok; w0 += kWin) {
        const int nw = min(kWin, kb1 - w0);
        if (!mbar_wait(acce_bar(accb), acc_phase[accb] ^ 1u, abort, g.wait_limit_ns)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem_base + uint32_t(accb * TN);
        int st = stage;
        uint32_t ph = phase;
        for (int q = 0; q < nw; ++q) {
          if (!mbar_wait(full_bar(st), ph, abort, g.wait_limit_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = base + st * STAGE_BYTES;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t ah = umma_desc_sw128(sa + kk * 32);
            const uint64_t al = umma_desc_sw128(sa + A_PLANE + kk * 32);
            const uint64_t bh = umma_desc_sw128(sa + 2 * A_PLANE + kk * 32);
            const uint64_t bl = umma_desc_sw128(sa + 2 * A_PLANE + B_PLANE + kk * 32);
            umma_tf32_pair(d, ah, bl, (q > 0 || kk > 0) ? 1u : 0u);
            umma_tf32_pair(d, al, bh, 1u);
          }
          if (++st == STAGES) {
            st = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
        for (int q = 0; q < nw; ++q) {
          const uint32_t sa = base + stage * STAGE_BYTES;
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            umma_tf32_pair(d, umma_desc_sw128(sa + kk * 32),
                           umma_desc_sw128(sa + 2 * A_PLANE + kk * 32), 1u);
          umma_commit_pair(empty_bar(stage));
          if (++stage == STAGES) {
            stage = 0;
            phase ^= 1u;
          }
        }
        umma_commit_pair(accf_bar(accb));
        acc_phase[accb] ^= 1u;
        accb ^= 1;
      }
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
  } else if (warp >= 2) {
    // ---- epilogue (both CTAs). Warp w reads TMEM lanes 32 (w % 4) .. +31
    // (its hardware lane quarter); warps 2-5 take columns 0-63 of the tile,
    // warps 6-9 columns 64-127. Each window's FP32 result is loaded, the
    // accumulator released at once, and the values added (round to nearest)
    // to a register sum of kFold windows; every kFold windows that sum is
    // folded into the double-float TMEM sum with 2Sum.
    const int quarter = warp & 3;
    const int col_lo = ((warp - 2) >> 2) * (TN / 2);
    const int row = int(rank) * 128 + quarter * 32 + lane;
    const uint32_t lane_addr = tmem_base + (uint32_t(quarter * 32) << 16);
    uint32_t acc_phase[2] = {0, 0};
    int accb = 0;
    bool ok = true;
    for (int u = pair; u < g.total_units && ok; u += npairs) {
      int sc, tm, tn;
      unit_of(u, sc, tm, tn);
      const int kb0 = sc * g.super_blocks, kb1 = min(g.kblocks, kb0 + g.super_blocks);
      const int i = tm * 256 + row;
      float mid[TN / 2];
#pragma unroll
      for (int c = 0; c < TN / 2; ++c) mid[c] = 0.0f;
      bool first_fold = true;
      int wi = 0;
      for (int w0 = kb0; w0 < kb1; w0 += kWin, ++wi) {
        // warp-uniform: the TMEM loads and the warp's arrival below are collective
        if (!__all_sync(0xffffffffu,
                        mbar_wait(accf_bar(accb), acc_phase[accb], abort, g.wait_limit_ns))) {
          ok = false;
          break;
        }
        tc_fence_after();
        static_assert(TN / 64 == 2, "two 32-column loads per warp and window");
        {
          uint32_t a0[32], a1[32];  // both loads in flight, one wait
          tmem_ld32_nowait(lane_addr + uint32_t(accb * TN + col_lo), a0);
          tmem_ld32_nowait(lane_addr + uint32_t(accb * TN + col_lo + 32), a1);
          tmem_wait_ld();
#pragma unroll
          for (int cc = 0; cc < 32; ++cc) {
            mid[cc] = __fadd_rn(mid[cc], __uint_as_float(a0[cc]));
            mid[32 + cc] = __fadd_rn(mid[32 + cc], __uint_as_float(a1[cc]));
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive_remote(map_to_rank(acce_bar(accb), 0));
        acc_phase[accb] ^= 1u;
        accb ^= 1;

        const bool last = w0 + kWin >= kb1;
        if (!last && (wi % kFold) != kFold - 1) continue;
#pragma unroll
        for (int q = 0; q < TN / 64; ++q) {
          const int c0 = col_lo + 32 * q;
          uint32_t h[32], l[32];
          if (!first_fold) {
            tmem_ld32_nowait(lane_addr + uint32_t(2 * TN + c0), h);
            tmem_ld32_nowait(lane_addr + uint32_t(3 * TN + c0), l);
            tmem_wait_ld();
          }
#pragma unroll
          for (int cc = 0; cc < 32; ++cc) {
            if (first_fold) {
              h[cc] = __float_as_uint(mid[32 * q + cc]);
              l[cc] = 0u;
            } else {
              float t, e;
              two_sum(__uint_as_float(h[cc]), mid[32 * q + cc], t, e);
              h[cc] = __float_as_uint(t);
              l[cc] = __float_as_uint(__fadd_rn(__uint_as_float(l[cc]), e));
            }
            mid[32 * q + cc] = 0.0f;
          }
          if (last) {
            if (i < g.m) {
              double* Pu = g.P + int64_t(sc) * g.nb * g.m;
#pragma unroll
              for (int cc = 0; cc < 32; ++cc) {
                const int j = tn * TN + c0 + cc;
                if (j < g.nb)
                  Pu[int64_t(j) * g.m + i] =
                      double(__uint_as_float(h[cc])) + double(__uint_as_float(l[cc]));
              }
            }
          } else {
            tmem_st32(lane_addr + uint32_t(2 * TN + c0), h);
            tmem_st32(lane_addr + uint32_t(3 * TN + c0), l);
          }
        }
        tmem_wait_st();
        first_fold = false;
      }
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

// C(i, j) <- alpha * sum_s P[s] + beta * C(i, j); complex: real part from row j
// of the real-form result, imaginary part from row n + j.
template <int DT>
__global__ void tf3_reduce(const double* __restrict__ P, int nsuper, int m, int n, int nb,
                           void* C, int64_t ldc, double alr, double ali, double ber, double bei,
                           int fill, int64_t ro, int64_t co, int tile_m, int tile_n) {
  constexpr bool CPLX = dtype_is_complex(DT);
  const int64_t total = int64_t(m) * n;
  const int64_t plane = int64_t(nb) * m;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int i = int(idx % m), j = int(idx / m);
    if (fill != 0) {
      const int64_t ti = (i / tile_m) * int64_t(tile_m), tj = (j / tile_n) * int64_t(tile_n);
      if (!tile_is_active(fill, ti, tj, ::min((int64_t)tile_m, (int64_t)m - ti),
                          ::min((int64_t)tile_n, (int64_t)n - tj), ro, co))
        continue;
    }
    double xr = 0.0, xi = 0.0;
    for (int s = 0; s < nsuper; ++s) {
      xr += P[s * plane + int64_t(j) * m + i];
      if (CPLX) xi += P[s * plane + int64_t(n + j) * m + i];
    }
    double outr = alr * xr - ali * xi, outi = alr * xi + ali * xr;
    const bool read_c = (ber != 0.0 || bei != 0.0);
    const int64_t ci = i + int64_t(j) * ldc;
    if constexpr (CPLX) {
      float2* c = static_cast<float2*>(C) + ci;
      if (read_c) {
        const float2 old = *c;
        outr += ber * double(old.x) - bei * double(old.y);
        outi += ber * double(old.y) + bei * double(old.x);
      }
      *c = make_float2(float(outr), float(outi));
    } else {
      float* c = static_cast<float*>(C) + ci;
      *c = float(read_c ? fma(ber, double(*c), outr) : outr);
    }
  }
}

struct Layout {
  int64_t K2, kp;
  int rowsA, rowsB, nb, nsuper, super_blocks;
  size_t off_Ah, off_Al, off_Bh, off_Bl, off_P, off_status, off_tiles, total;
};

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    sms = 148;
  }
  return sms;
}

// Number of k super-chunks: each adds one FP64 partial plane (written by the
// GEMM, read by the reduction) but evens out the last round of work units
// over the CTA pairs. Minimises the modelled time
//   (3 TF32 products at 0.5 PFLOP/s) / (balance of units over pairs)
//   + partial traffic at 6 TB/s.
int choose_splits(int64_t kblocks, int tiles, int pairs, int64_t m, int64_t nb) {
  const int64_t max_s = std::max<int64_t>(
      1, std::min<int64_t>(256, (kblocks + kMinSuperBlocks - 1) / kMinSuperBlocks));
  const double t_mma = 3.0 * 2.0 * double(m) * double(nb) * double(kblocks) * BKF / 5e14;
  const double t_plane = 2.0 * 8.0 * double(m) * double(nb) / 6e12;
  int best = 1;
  double best_t = 1e300;
  for (int64_t s = 1; s <= max_s; ++s) {
    const int64_t units = int64_t(tiles) * s;
    const int64_t rounds = (units + pairs - 1) / pairs;
    const double t = t_mma * double(rounds * pairs) / double(units) + t_plane * double(s);
    if (t < best_t * 0.999) {
      best_t = t;
      best = int(s);
    }
  }
  return best;
}

Layout layout_of(const GemmProblem& p) {
  Layout L{};
  const bool cplx = dtype_is_complex(p.dtype);
  L.K2 = cplx ? 2 * p.k : p.k;
  L.kp = (L.K2 + BKF - 1) / BKF * BKF;
  L.rowsA = int(p.m);
  L.rowsB = int(p.n);
  L.nb = cplx ? int(2 * p.n) : int(p.n);
  const int64_t kblocks = L.kp / BKF;
  const int tiles = ((L.rowsA + 255) / 256) * ((L.nb + TN - 1) / TN);
  int s = choose_splits(kblocks, tiles, std::max(1, sm_count() / 2), L.rowsA, L.nb);
  if (const char* v = std::getenv("SPLAB_TF32X3_SPLITS")) {  // tuning override
    const int f = std::atoi(v);
    if (f > 0) s = int(std::min<int64_t>(f, kblocks > 0 ? kblocks : 1));
  }
  L.super_blocks = int(std::max<int64_t>(1, (kblocks + s - 1) / s));
  L.nsuper = int(std::max<int64_t>(1, (kblocks + L.super_blocks - 1) / L.super_blocks));
  size_t off = 0;
  L.off_Ah = off;
  off = al256(off + sizeof(float) * size_t(L.rowsA) * L.kp);
  L.off_Al = off;
  off = al256(off + sizeof(float) * size_t(L.rowsA) * L.kp);
  L.off_Bh = off;
  off = al256(off + sizeof(float) * size_t(L.nb) * L.kp);
  L.off_Bl = off;
  off = al256(off + sizeof(float) * size_t(L.nb) * L.kp);
  L.off_P = off;
  off = al256(off + sizeof(double) * size_t(L.nsuper) * L.nb * L.rowsA);
  L.off_status = off;
  off = al256(off + 256);
  L.off_tiles = off;
  off = al256(off + sizeof(int) * size_t((L.rowsA + 255) / 256) * ((L.nb + TN - 1) / TN));
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

bool make_map(CUtensorMap* map, void* base, int64_t kp, int64_t rows, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {cuuint64_t(kp), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(kp) * sizeof(float)};
  cuuint32_t box[2] = {cuuint32_t(BKF), box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace tf3

bool tf32x3_supported(const GemmProblem& p) {
  return (p.dtype == kR32 || p.dtype == kC32) && p.opA != 0 && p.opB == 0 &&
         p.m <= (1 << 24) && p.n <= (1 << 23);
}

size_t tf32x3_workspace_bytes(const GemmProblem& p) {
  if (p.m <= 0 || p.n <= 0) return 0;
  return tf3::layout_of(p).total;
}

cudaError_t tf32x3_gemm(const GemmProblem& p, void* ws, size_t ws_bytes, cudaStream_t st) {
  using namespace tf3;
  if (!tf32x3_supported(p)) return cudaErrorNotSupported;
  if (p.m <= 0 || p.n <= 0) return cudaSuccess;
  const Layout L = layout_of(p);
  if (!ws || ws_bytes < L.total) return cudaErrorInvalidValue;
  const bool cplx = dtype_is_complex(p.dtype);
  char* w = static_cast<char*>(ws);
  float* Ah = reinterpret_cast<float*>(w + L.off_Ah);
  float* Al = reinterpret_cast<float*>(w + L.off_Al);
  float* Bh = reinterpret_cast<float*>(w + L.off_Bh);
  float* Bl = reinterpret_cast<float*>(w + L.off_Bl);
  double* P = reinterpret_cast<double*>(w + L.off_P);
  int* status = reinterpret_cast<int*>(w + L.off_status);
  cudaError_t e;
  phase_mark(0, false, st);
  if (p.k > 0) {
    const int64_t ldA = cplx ? 2 * p.lda : p.lda, ldB = cplx ? 2 * p.ldb : p.ldb;
    const int64_t groups = L.kp / 4;
    tf3_split<<<unsigned((L.rowsA * groups + 255) / 256), 256, 0, st>>>(
        static_cast<const float*>(p.A), ldA, L.K2, L.rowsA, L.kp, 0, 1, Ah, Al);
    tf3_split<<<unsigned((L.rowsB * groups + 255) / 256), 256, 0, st>>>(
        static_cast<const float*>(p.B), ldB, L.K2, L.rowsB, L.kp, cplx ? 1 : 0,
        p.opA == 2 ? -1 : 1, Bh, Bl);
  }
  cudaMemsetAsync(status, 0, sizeof(int), st);
  phase_mark(0, true, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;

  phase_mark(1, false, st);
  int nsuper = L.nsuper;
  if (p.k > 0) {
    CUtensorMap mAh, mAl, mBh, mBl;
    if (!make_map(&mAh, Ah, L.kp, L.rowsA, 128) || !make_map(&mAl, Al, L.kp, L.rowsA, 128) ||
        !make_map(&mBh, Bh, L.kp, L.nb, TN / 2) || !make_map(&mBl, Bl, L.kp, L.nb, TN / 2))
      return cudaErrorNotSupported;
    GemmParams g{};
    g.m = L.rowsA;
    g.nb = L.nb;
    g.kblocks = int(L.kp / BKF);
    g.super_blocks = L.super_blocks;
    g.nsuper = L.nsuper;
    g.tiles_m = (L.rowsA + 255) / 256;
    g.tiles_n = (L.nb + TN - 1) / TN;
    g.P = P;
    g.status = status;
    g.wait_limit_ns = kWaitLimitNs;
    if (const char* v = std::getenv("SPLAB_TF32X3_STALL_TEST")) {
      // test hook for the failure path: no copies are issued, every wait runs
      // into a 50 ms bound, the kernel reports SPLAB_ERR_TIMEOUT and returns
      if (v[0] == '1') {
        g.stall_test = 1;
        g.wait_limit_ns = 50000000ull;
      }
    }
    int ntiles = g.tiles_m * g.tiles_n;
    if (p.fill_mode != 0) {
      const int rt_m = 128, rt_n = 128;  // reconstruction tiles of C
      std::vector<int> act;
      for (int tn = 0; tn < g.tiles_n; ++tn)
        for (int tm = 0; tm < g.tiles_m; ++tm) {
          const int64_t r0 = int64_t(tm) * 256, r1 = std::min<int64_t>(r0 + 256, L.rowsA);
          const int64_t b0 = int64_t(tn) * TN, b1 = std::min<int64_t>(b0 + TN, L.nb);
          int64_t cr[2][2];
          int ncr = 0;
          if (!cplx) {
            cr[ncr][0] = b0;
            cr[ncr++][1] = b1;
          } else {
            if (b0 < p.n) {
              cr[ncr][0] = b0;
              cr[ncr++][1] = std::min<int64_t>(b1, p.n);
            }
            if (b1 > p.n) {
              cr[ncr][0] = std::max<int64_t>(b0, p.n) - p.n;
              cr[ncr++][1] = b1 - p.n;
            }
          }
          bool on = false;
          for (int q = 0; q < ncr && !on; ++q)
            for (int64_t ti = (r0 / rt_m) * rt_m; ti < r1 && !on; ti += rt_m)
              for (int64_t tj = (cr[q][0] / rt_n) * rt_n; tj < cr[q][1] && !on; tj += rt_n)
                on = tile_is_active(p.fill_mode, ti, tj, std::min<int64_t>(rt_m, p.m - ti),
                                    std::min<int64_t>(rt_n, p.n - tj), p.fill_ro, p.fill_co);
          if (on) act.push_back(tm + tn * g.tiles_m);
        }
      if (act.empty()) act.push_back(0);
      int* dt = reinterpret_cast<int*>(w + L.off_tiles);
      if ((e = cudaMemcpyAsync(dt, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice,
                               st)) != cudaSuccess)
        return e;
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
      g.active = dt;
      g.n_active = int(act.size());
      ntiles = g.n_active;
    }
    g.total_units = ntiles * g.nsuper;
    if ((e = set_dynamic_smem(reinterpret_cast<const void*>(tf3_gemm_pair), SMEM)) !=
        cudaSuccess)
      return e;
    const int pairs = std::max(1, std::min(g.total_units, sm_count() / 2));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(unsigned(2 * pairs));
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if ((e = cudaLaunchKernelEx(&cfg, tf3_gemm_pair, mAh, mAl, mBh, mBl, g)) != cudaSuccess)
      return e;
  } else {
    nsuper = 0;
  }
  phase_mark(1, true, st);

  phase_mark(2, false, st);
  const int64_t total = p.m * p.n;
  const unsigned blocks = unsigned(std::min<int64_t>((total + 255) / 256, 148 * 32));
  if (cplx)
    tf3_reduce<kC32><<<blocks, 256, 0, st>>>(P, nsuper, L.rowsA, int(p.n), L.nb, p.C, p.ldc,
                                             p.alpha[0], p.alpha[1], p.beta[0], p.beta[1],
                                             p.fill_mode, p.fill_ro, p.fill_co, 128, 128);
  else
    tf3_reduce<kR32><<<blocks, 256, 0, st>>>(P, nsuper, L.rowsA, int(p.n), L.nb, p.C, p.ldc,
                                             p.alpha[0], p.alpha[1], p.beta[0], p.beta[1],
                                             p.fill_mode, p.fill_ro, p.fill_co, 128, 128);
  phase_mark(2, true, st);
  return cudaGetLastError();
}

int* tf32x3_status_ptr(const GemmProblem& p, void* ws) {
  return reinterpret_cast<int*>(static_cast<char*>(ws) + tf3::layout_of(p).off_status);
}

int tf32x3_status(const GemmProblem& p, void* ws, cudaStream_t st) {
  const tf3::Layout L = tf3::layout_of(p);
  int h = 0;
  cudaMemcpyAsync(&h, static_cast<char*>(ws) + L.off_status, sizeof(int), cudaMemcpyDeviceToHost,
                  st);
  cudaStreamSynchronize(st);
  return h;
}

}  // namespace splab
