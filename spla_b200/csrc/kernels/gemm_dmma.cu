// FP64 tensor-core contraction for the SPLA local path (sm_100a).
//
// C(m x n) <- alpha * op(A) * op(B) + beta * C for real/complex, float/double,
// with op in {N, T, C} on both operands: the single-rank work of pgemm_ssb
// (opA in {T, C}, opB = N: src/pgemm_ssb/pgemm_ssb_host.cpp:168-171),
// pgemm_sbs (N, N: src/pgemm_sbs/pgemm_sbs_host.cpp:179-183) and gemm()
// (src/gemm/gemm_gpu.cpp:59-174).
//
// tcgen05 has no f64 kind, so the FP64 tensor path is warp-level
// mma.sync.m8n8k4.f64 fed from a cp.async multi-stage shared-memory pipeline.
// Float inputs go through the same kernel: products of two floats are exact
// in double and the sums run in FP64, so the float result is the double-
// precision result rounded once.
//
// Split-K: the long dimension k is cut into `splits` ranges (grid.y). With one
// split the epilogue applies alpha/beta and writes C directly; otherwise each
// CTA writes its FP64 partial tile and splab_reduce_partials() sums the splits
// in a fixed order (deterministic) and applies alpha/beta. Every per-element
// FP64 chain is at most k/splits long and the splits are summed pairwise-free
// in order, which keeps the complex k=250000 case near 2e-15 relative error.
//
// Fill mode: tiles of C that do not intersect the requested triangle are
// skipped (C left unchanged), with the reference's block predicate
// (src/block_generation/block.hpp:58-66) applied per tile.
#include <cuda.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "../../../include/splab.h"
#include "gemm_dmma.cuh"

namespace splab {

template <int DT>
struct Elem;
template <>
struct Elem<kR64> {
  using S = double;
  static constexpr bool cplx = false;
};
template <>
struct Elem<kR32> {
  using S = float;
  static constexpr bool cplx = false;
};
template <>
struct Elem<kC64> {
  using S = double2;
  static constexpr bool cplx = true;
};
template <>
struct Elem<kC32> {
  using S = float2;
  static constexpr bool cplx = true;
};

__device__ __forceinline__ void to_re_im(double v, double& re, double& im) { re = v; im = 0.0; }
__device__ __forceinline__ void to_re_im(float v, double& re, double& im) {
  re = static_cast<double>(v);
  im = 0.0;
}
__device__ __forceinline__ void to_re_im(double2 v, double& re, double& im) { re = v.x; im = v.y; }
__device__ __forceinline__ void to_re_im(float2 v, double& re, double& im) {
  re = static_cast<double>(v.x);
  im = static_cast<double>(v.y);
}

// Copy one element (global -> shared) asynchronously, zero-filled when invalid.
template <typename S>
__device__ __forceinline__ void cp_elem(S* dst, const S* src, bool valid) {
  if constexpr (sizeof(S) == 4) {
    cp_async_4(dst, src, valid);
  } else if constexpr (sizeof(S) == 8) {
    cp_async_8(dst, src, valid);
  } else {
    cp_async_8(dst, src, valid);
    cp_async_8(reinterpret_cast<char*>(dst) + 8, reinterpret_cast<const char*>(src) + 8, valid);
  }
}

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// Row stride (in elements) of a staged operand tile, chosen so that the
// fragment reads of one mma.m8n8k4 are free of shared-memory bank conflicts.
template <int BYTES, bool KMAJ, int T, int BK>
struct SmemStride {
  static constexpr int value =
      KMAJ ? (BK + 4) : (BYTES == 4 ? T + 8 : (BYTES == 8 ? T + 4 : T + 2));
};

template <int DT_, bool AK_, bool BK_MAJ_, int BM_, int BN_, int BK_, int WM_, int WN_, int ST_>
struct DmmaCfg {
  static constexpr int DT = DT_;
  using S = typename Elem<DT>::S;
  static constexpr bool CPLX = Elem<DT>::cplx;
  static constexpr bool A_KMAJ = AK_;
  static constexpr bool B_KMAJ = BK_MAJ_;
  static constexpr int BM = BM_, BN = BN_, BK = BK_, WM = WM_, WN = WN_, STAGES = ST_;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int THREADS = 32 * WARPS_M * WARPS_N;
  static constexpr int SA = SmemStride<sizeof(S), A_KMAJ, BM, BK>::value;
  static constexpr int SB = SmemStride<sizeof(S), B_KMAJ, BN, BK>::value;
  static constexpr int A_ELEMS = A_KMAJ ? BM * SA : BK * SA;
  static constexpr int B_ELEMS = B_KMAJ ? BN * SB : BK * SB;
  static constexpr int STAGE_BYTES = (A_ELEMS + B_ELEMS) * int(sizeof(S));
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES;
  static_assert((BM * BK) % THREADS == 0 && (BN * BK) % THREADS == 0, "tile/threads");
  static_assert(BK % 4 == 0 && WM % 8 == 0 && WN % 8 == 0, "mma shape");
};

// Stage one T x BK operand tile. KMAJ: element (r, c) at X[(r0+r)*ld + k0+c];
// otherwise at X[(k0+c)*ld + r0+r]. Rows >= rows_total or k >= kend read zero.
template <typename S, bool KMAJ, int T, int BK, int STRIDE, int THREADS>
__device__ __forceinline__ void stage_tile(S* smem, const S* X, int64_t ld, int64_t r0,
                                           int64_t rows_total, int64_t k0, int64_t kend) {
  constexpr int ELEMS = T * BK;
#pragma unroll
  for (int i = 0; i < ELEMS / THREADS; ++i) {
    const int e = threadIdx.x + i * THREADS;
    int r, c;
    if constexpr (KMAJ) {
      c = e % BK;
      r = e / BK;
    } else {
      r = e % T;
      c = e / T;
    }
    const int64_t gr = r0 + r, gk = k0 + c;
    const bool valid = (gr < rows_total) && (gk < kend);
    const S* src = valid ? (KMAJ ? X + gr * ld + gk : X + gk * ld + gr) : X;
    S* dst = KMAJ ? smem + r * STRIDE + c : smem + c * STRIDE + r;
    cp_elem(dst, src, valid);
  }
}

template <typename S, bool KMAJ, int STRIDE>
__device__ __forceinline__ S frag_load(const S* smem, int row, int kidx) {
  return KMAJ ? smem[row * STRIDE + kidx] : smem[kidx * STRIDE + row];
}

// C[idx] <- alpha * x + beta * C[idx] over the dtype of C, reading C only if
// beta != 0 (BLAS semantics).
template <int DT>
__device__ __forceinline__ void store_alpha_beta_impl(void* C, int64_t idx, double xr, double xi,
                                                      double alr, double ali, double ber,
                                                      double bei) {
  double outr = alr * xr - ali * xi;
  double outi = alr * xi + ali * xr;
  const bool read_c = (ber != 0.0 || bei != 0.0);
  if constexpr (DT == kR64) {
    double* c = static_cast<double*>(C) + idx;
    *c = read_c ? fma(ber, *c, outr) : outr;
  } else if constexpr (DT == kR32) {
    float* c = static_cast<float*>(C) + idx;
    *c = static_cast<float>(read_c ? fma(ber, static_cast<double>(*c), outr) : outr);
  } else if constexpr (DT == kC64) {
    double2* c = static_cast<double2*>(C) + idx;
    if (read_c) {
      const double2 v = *c;
      outr += ber * v.x - bei * v.y;
      outi += ber * v.y + bei * v.x;
    }
    *c = make_double2(outr, outi);
  } else {
    float2* c = static_cast<float2*>(C) + idx;
    if (read_c) {
      const float2 v = *c;
      outr += ber * double(v.x) - bei * double(v.y);
      outi += ber * double(v.y) + bei * double(v.x);
    }
    *c = make_float2(static_cast<float>(outr), static_cast<float>(outi));
  }
}

// One CTA tile (tile index -> (tm, tn), column of tiles fastest) over the
// k-range of split `split`.
template <class Cfg>
__device__ __forceinline__ void dmma_tile(const DmmaParams& p, int64_t tile, int split,
                                          unsigned char* smem_raw) {
  using S = typename Cfg::S;
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, WM = Cfg::WM, WN = Cfg::WN;
  constexpr int FM = WM / 8, FN = WN / 8, STAGES = Cfg::STAGES;
  constexpr bool CPLX = Cfg::CPLX;

  S* smem = reinterpret_cast<S*>(smem_raw);

  const int64_t tiles_m = (p.m + BM - 1) / BM;
  const int64_t tm = tile % tiles_m, tn = tile / tiles_m;
  const int64_t m0 = tm * BM, n0 = tn * BN;
  if (!tile_is_active(p.fill_mode, m0, n0, ::min((int64_t)BM, p.m - m0),
                      ::min((int64_t)BN, p.n - n0), p.fill_ro, p.fill_co))
    return;

  const int64_t kbeg = static_cast<int64_t>(split) * p.k_per_split;
  const int64_t kend = min(p.k, kbeg + p.k_per_split);
  const int nkt = kend > kbeg ? static_cast<int>((kend - kbeg + BK - 1) / BK) : 0;

  const S* A = static_cast<const S*>(p.A);
  const S* B = static_cast<const S*>(p.B);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp % Cfg::WARPS_M, wn = warp / Cfg::WARPS_M;
  const int g = lane >> 2, t = lane & 3;
  const unsigned long long maskA = p.conj_a ? 0x8000000000000000ull : 0ull;
  const unsigned long long maskB = p.conj_b ? 0x8000000000000000ull : 0ull;
  constexpr unsigned long long kNeg = 0x8000000000000000ull;

  double accr[FM][FN][2];
  double acci[CPLX ? FM : 1][CPLX ? FN : 1][2];
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) {
      accr[i][j][0] = accr[i][j][1] = 0.0;
      if constexpr (CPLX) acci[i][j][0] = acci[i][j][1] = 0.0;
    }

  auto stage_ptr_a = [&](int s) { return smem + s * (Cfg::A_ELEMS + Cfg::B_ELEMS); };
  auto stage_ptr_b = [&](int s) { return smem + s * (Cfg::A_ELEMS + Cfg::B_ELEMS) + Cfg::A_ELEMS; };
  auto load_stage = [&](int s, int64_t k0) {
    stage_tile<S, Cfg::A_KMAJ, BM, BK, Cfg::SA, Cfg::THREADS>(stage_ptr_a(s), A, p.lda, m0, p.m,
                                                             k0, kend);
    stage_tile<S, Cfg::B_KMAJ, BN, BK, Cfg::SB, Cfg::THREADS>(stage_ptr_b(s), B, p.ldb, n0, p.n,
                                                             k0, kend);
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nkt) load_stage(s, kbeg + static_cast<int64_t>(s) * BK);
    cp_async_commit();
  }

  for (int kt = 0; kt < nkt; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int pf = kt + STAGES - 1;
    if (pf < nkt) load_stage(pf % STAGES, kbeg + static_cast<int64_t>(pf) * BK);
    cp_async_commit();

    const S* As = stage_ptr_a(kt % STAGES);
    const S* Bs = stage_ptr_b(kt % STAGES);
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double ar[FM], ai[FM], ain[FM], br[FN], bi[FN];
#pragma unroll
      for (int i = 0; i < FM; ++i) {
        double re, im;
        to_re_im(frag_load<S, Cfg::A_KMAJ, Cfg::SA>(As, wm * WM + i * 8 + g, kk + t), re, im);
        ar[i] = re;
        ai[i] = xor_sign(im, maskA);
        ain[i] = xor_sign(ai[i], kNeg);
      }
#pragma unroll
      for (int j = 0; j < FN; ++j) {
        double re, im;
        to_re_im(frag_load<S, Cfg::B_KMAJ, Cfg::SB>(Bs, wn * WN + j * 8 + g, kk + t), re, im);
        br[j] = re;
        bi[j] = xor_sign(im, maskB);
      }
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) {
          dmma_8x8x4(accr[i][j][0], accr[i][j][1], ar[i], br[j]);
          if constexpr (CPLX) {
            dmma_8x8x4(accr[i][j][0], accr[i][j][1], ain[i], bi[j]);
            dmma_8x8x4(acci[i][j][0], acci[i][j][1], ar[i], bi[j]);
            dmma_8x8x4(acci[i][j][0], acci[i][j][1], ai[i], br[j]);
          }
        }
    }
  }
  cp_async_wait<0>();

  // Epilogue: element (i, j) of the warp's sub-tile (fi, fj, e).
#pragma unroll
  for (int fi = 0; fi < FM; ++fi) {
    const int64_t i = m0 + wm * WM + fi * 8 + g;
    if (i >= p.m) continue;
#pragma unroll
    for (int fj = 0; fj < FN; ++fj) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int64_t j = n0 + wn * WN + fj * 8 + 2 * t + e;
        if (j >= p.n) continue;
        const double xr = accr[fi][fj][e];
        const double xi = CPLX ? acci[CPLX ? fi : 0][CPLX ? fj : 0][e] : 0.0;
        if (p.partial) {
          const int64_t idx = static_cast<int64_t>(split) * p.m * p.n + j * p.m + i;
          if constexpr (CPLX) {
            reinterpret_cast<double2*>(p.P)[idx] = make_double2(xr, xi);
          } else {
            reinterpret_cast<double*>(p.P)[idx] = xr;
          }
        } else {
          store_alpha_beta_impl<Cfg::DT>(p.C, i + j * p.ldc, xr, xi, p.alpha_r, p.alpha_i,
                                            p.beta_r, p.beta_i);
        }
      }
    }
  }
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS) dmma_gemm_kernel(DmmaParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  dmma_tile<Cfg>(p, blockIdx.x, int(blockIdx.y), smem_raw);
}

// Persistent grouped form: CTAs walk a list of (instance, tile, split) work
// items of many independent problems of one configuration (one launch for a
// whole batch). Items are pre-sorted by the host (longest first).
template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS)
    dmma_gemm_grouped_kernel(const DmmaParams* __restrict__ params, const int4* __restrict__ items,
                             int n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 w = items[it];
    __syncthreads();  // the previous item's fragments are no longer read
    dmma_tile<Cfg>(params[w.x], w.y, w.z, smem_raw);
  }
}

// Sum the FP64 split-K partials of each element in split order, then
// C <- alpha * sum + beta * C. Elements of tiles outside the fill triangle are
// left untouched (the same tile predicate as the GEMM kernel).
template <int DT>
__global__ void reduce_partials_kernel(const void* __restrict__ P, int splits, int64_t m,
                                       int64_t n, void* C, int64_t ldc, double alr, double ali,
                                       double ber, double bei, int fill_mode, int64_t ro,
                                       int64_t co, int tile_m, int tile_n) {
  constexpr bool CPLX = dtype_is_complex(DT);
  const int64_t total = m * n;
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx % m, j = idx / m;
    if (fill_mode != 0) {
      const int64_t ti = (i / tile_m) * tile_m, tj = (j / tile_n) * tile_n;
      if (!tile_is_active(fill_mode, ti, tj, ::min((int64_t)tile_m, m - ti),
                          ::min((int64_t)tile_n, n - tj), ro, co))
        continue;
    }
    double sr = 0.0, si = 0.0;
    if constexpr (CPLX) {
      const double2* q = static_cast<const double2*>(P) + idx;
      for (int s = 0; s < splits; ++s) {
        const double2 v = q[s * total];
        sr += v.x;
        si += v.y;
      }
    } else {
      const double* q = static_cast<const double*>(P) + idx;
      for (int s = 0; s < splits; ++s) sr += q[s * total];
    }
    store_alpha_beta_impl<DT>(C, i + j * ldc, sr, si, alr, ali, ber, bei);
  }
}

// ---------------------------------------------------------------------------
// Host side: configuration per (dtype, operand layouts), split selection.

namespace {

template <int DT, bool AK, bool BKM>
struct CfgFor;
// complex: 64x64 CTA tile, 2x2 warps of 32x32, BK = 8 complex
template <bool AK, bool BKM>
struct CfgFor<kC64, AK, BKM> {
  using type = DmmaCfg<kC64, AK, BKM, 64, 64, 8, 32, 32, 3>;
};
template <bool AK, bool BKM>
struct CfgFor<kC32, AK, BKM> {
  using type = DmmaCfg<kC32, AK, BKM, 64, 64, 8, 32, 32, 3>;
};
// real: 128x64 CTA tile, 4x2 warps of 32x32, BK = 16
template <bool AK, bool BKM>
struct CfgFor<kR64, AK, BKM> {
  using type = DmmaCfg<kR64, AK, BKM, 128, 64, 16, 32, 32, 3>;
};
template <bool AK, bool BKM>
struct CfgFor<kR32, AK, BKM> {
  using type = DmmaCfg<kR32, AK, BKM, 128, 64, 16, 32, 32, 3>;
};

// Larger-tile variant that the batch autotuner measures beside the default:
// complex 128x64 (8 warps), real 128x128 (16 warps); same k-step as CfgFor.
template <int DT, bool AK, bool BKM>
struct CfgWide;
template <bool AK, bool BKM>
struct CfgWide<kC64, AK, BKM> {
  using type = DmmaCfg<kC64, AK, BKM, 128, 64, 8, 32, 32, 3>;
};
template <bool AK, bool BKM>
struct CfgWide<kC32, AK, BKM> {
  using type = DmmaCfg<kC32, AK, BKM, 128, 64, 8, 32, 32, 3>;
};
template <bool AK, bool BKM>
struct CfgWide<kR64, AK, BKM> {
  using type = DmmaCfg<kR64, AK, BKM, 128, 128, 16, 32, 32, 3>;
};
template <bool AK, bool BKM>
struct CfgWide<kR32, AK, BKM> {
  using type = DmmaCfg<kR32, AK, BKM, 128, 128, 16, 32, 32, 3>;
};
constexpr int kBatchTileVariants = 2;

template <class Cfg>
int occupancy() {
  static int occ = -1;
  set_dynamic_smem(reinterpret_cast<const void*>(dmma_gemm_kernel<Cfg>), Cfg::SMEM_BYTES);
  if (occ < 0) {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, dmma_gemm_kernel<Cfg>, Cfg::THREADS,
                                                      Cfg::SMEM_BYTES) != cudaSuccess ||
        o < 1)
      o = 1;
    occ = o;
  }
  return occ;
}

template <class Cfg>
DmmaPlan plan_for(const GemmProblem& pr, int num_sms, int force_splits) {
  DmmaPlan plan{Cfg::BM, Cfg::BN, 1, Cfg::BK, 0};
  if (pr.k <= 0) return plan;  // C <- beta C only: one pass, no partials
  const int64_t tiles = ((pr.m + Cfg::BM - 1) / Cfg::BM) * ((pr.n + Cfg::BN - 1) / Cfg::BN);
  const int64_t slots = int64_t(num_sms) * occupancy<Cfg>();
  const double flop_per_k = double(Cfg::BM) * Cfg::BN * (Cfg::CPLX ? 8.0 : 2.0);
  const double slot_rate = 37e12 / double(slots);  // FP64 tensor rate per resident CTA
  const double esz = Cfg::CPLX ? 16.0 : 8.0;
  int best_s = 1;
  if (force_splits > 0) {
    best_s = force_splits;
  } else {
    double best_t = 1e300;
    const int64_t s_max = std::max<int64_t>(1, std::min<int64_t>(4096, pr.k / (8 * Cfg::BK)));
    for (int64_t s = 1; s <= s_max; ++s) {
      const int64_t kps = ((pr.k + s - 1) / s + Cfg::BK - 1) / Cfg::BK * Cfg::BK;
      const int64_t s_eff = (pr.k + kps - 1) / kps;
      if (s_eff != s) continue;
      const double waves = double((tiles * s + slots - 1) / slots);
      const double t = waves * double(kps) * flop_per_k / slot_rate +
                       (s > 1 ? double(s) * pr.m * pr.n * esz * 2.0 / 6.0e12 : 0.0) +
                       (s > 1 ? 4e-6 : 0.0);
      if (t < best_t * 0.995) {
        best_t = t;
        best_s = int(s);
      }
    }
  }
  int64_t kps = ((pr.k + best_s - 1) / best_s + Cfg::BK - 1) / Cfg::BK * Cfg::BK;
  if (kps < 1) kps = Cfg::BK;
  plan.splits = int(std::max<int64_t>(1, (pr.k + kps - 1) / kps));
  plan.k_per_split = kps;
  plan.workspace_bytes = plan.splits > 1 ? size_t(plan.splits) * pr.m * pr.n * size_t(esz) : 0;
  return plan;
}

template <class Cfg>
cudaError_t launch_cfg(const GemmProblem& pr, const DmmaPlan& plan, void* ws, cudaStream_t st) {
  occupancy<Cfg>();  // also sets the dynamic shared memory attribute
  DmmaParams p{};
  p.A = pr.A;
  p.B = pr.B;
  p.C = pr.C;
  p.P = ws;
  p.lda = pr.lda;
  p.ldb = pr.ldb;
  p.ldc = pr.ldc;
  p.m = pr.m;
  p.n = pr.n;
  p.k = pr.k;
  p.k_per_split = plan.k_per_split;
  p.alpha_r = pr.alpha[0];
  p.alpha_i = pr.alpha[1];
  p.beta_r = pr.beta[0];
  p.beta_i = pr.beta[1];
  p.conj_a = pr.opA == 2;
  p.conj_b = pr.opB == 2;
  p.partial = plan.splits > 1;
  p.fill_mode = pr.fill_mode;
  p.fill_ro = pr.fill_ro;
  p.fill_co = pr.fill_co;
  const int64_t tiles = ((pr.m + Cfg::BM - 1) / Cfg::BM) * ((pr.n + Cfg::BN - 1) / Cfg::BN);
  dim3 grid(unsigned(tiles), unsigned(plan.splits));
  phase_mark(0, false, st);
  dmma_gemm_kernel<Cfg><<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(p);
  phase_mark(0, true, st);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || plan.splits == 1) return e;
  phase_mark(1, false, st);
  e = reduce_partials(pr, ws, plan.splits, Cfg::BM, Cfg::BN, st);
  phase_mark(1, true, st);
  return e;
}

template <int DT, class F>
auto with_cfg(const GemmProblem& pr, F&& f) {
  const bool ak = pr.opA != 0;   // op(A) = A^T / A^H: A is k x m, k contiguous
  const bool bk = pr.opB == 0;   // op(B) = B: B is k x n, k contiguous
  if (ak && bk) return f(typename CfgFor<DT, true, true>::type{});
  if (ak && !bk) return f(typename CfgFor<DT, true, false>::type{});
  if (!ak && bk) return f(typename CfgFor<DT, false, true>::type{});
  return f(typename CfgFor<DT, false, false>::type{});
}

template <class F>
auto dispatch(const GemmProblem& pr, F&& f) {
  switch (pr.dtype) {
    case kR32: return with_cfg<kR32>(pr, f);
    case kR64: return with_cfg<kR64>(pr, f);
    case kC32: return with_cfg<kC32>(pr, f);
    default: return with_cfg<kC64>(pr, f);
  }
}

}  // namespace

DmmaPlan dmma_plan(const GemmProblem& pr, int num_sms, int force_splits) {
  return dispatch(pr, [&](auto cfg) {
    return plan_for<decltype(cfg)>(pr, num_sms, force_splits);
  });
}

cudaError_t dmma_gemm(const GemmProblem& pr, const DmmaPlan& plan, void* ws, cudaStream_t st) {
  if (pr.m <= 0 || pr.n <= 0) return cudaSuccess;
  return dispatch(pr, [&](auto cfg) { return launch_cfg<decltype(cfg)>(pr, plan, ws, st); });
}

cudaError_t reduce_partials(const GemmProblem& pr, const void* P, int splits, int tile_m,
                            int tile_n, cudaStream_t st) {
  const int64_t total = pr.m * pr.n;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>((total + threads - 1) / threads, 148 * 16);
  auto go = [&](auto kern) {
    kern<<<unsigned(blocks), threads, 0, st>>>(P, splits, pr.m, pr.n, pr.C, pr.ldc, pr.alpha[0],
                                               pr.alpha[1], pr.beta[0], pr.beta[1], pr.fill_mode,
                                               pr.fill_ro, pr.fill_co, tile_m, tile_n);
    return cudaGetLastError();
  };
  switch (pr.dtype) {
    case kR32: return go(reduce_partials_kernel<kR32>);
    case kR64: return go(reduce_partials_kernel<kR64>);
    case kC32: return go(reduce_partials_kernel<kC32>);
    default: return go(reduce_partials_kernel<kC64>);
  }
}


// ---------------------------------------------------------------------------
// Allocation-free variant of the FP64 contraction.
//
// For callers that must not allocate device memory themselves or through
// this library: applications whose device memory is owned by a framework
// allocator that has to account for every byte, processes running against a
// hard device-memory cap, and latency-critical loops that cannot afford the
// implicit device synchronisation of cudaMalloc / cudaFree. The split-K
// partials live in one file-scope device array of SPLAB_NOALLOC_SCRATCH_BYTES
// that every GPU loading this library holds until the process exits.
//
// The array's host-side symbol is only a stand-in: its device address is
// looked up with cudaGetSymbolAddress, once per device, by the first call on
// that device (with that device current), and again after a device reset
// (a new context). Make that first call before any stream capture. All calls share the array and it keeps the last call's
// contents; nothing in it has to start at zero (every split overwrites its
// partial tile before the reduction reads it). Calls whose execution overlaps
// on the GPU (different streams, or different host threads) race on the
// array and must be serialised by the caller.

static __device__ __align__(256) unsigned char noalloc_scratch[SPLAB_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex noalloc_mutex;
struct NoallocSlot {
  unsigned long long context_id = 0;  // the CUDA context the address belongs to
  void* ptr = nullptr;
};
NoallocSlot noalloc_slot[64];

// Unique id of the calling thread's current CUDA context, 0 when it cannot be
// read. A device reset (cudaDeviceReset) destroys the context and the module
// with the array; the next context loads the module anew and the array may
// sit at another address, so the address is cached per device AND context.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  if (get_current(&c) != CUDA_SUCCESS || c == nullptr) return 0;
  unsigned long long id = 0;
  return get_id(c, &id) == CUDA_SUCCESS ? id : 0;
}

// Device address of noalloc_scratch on the current device, looked up once per
// device and context (with that device current); the lookup allocates nothing.
cudaError_t noalloc_scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(noalloc_mutex);
  NoallocSlot& slot = noalloc_slot[dev];
  const unsigned long long id = current_context_id();
  if (slot.ptr == nullptr || id == 0 || id != slot.context_id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, noalloc_scratch);
    if (e != cudaSuccess) return e;
    slot.ptr = p;
    slot.context_id = current_context_id();  // the lookup made the context current
  }
  *out = slot.ptr;
  return cudaSuccess;
}
}  // namespace

int dmma_gemm_noalloc(const GemmProblem& pr, int num_sms, cudaStream_t st) {
  if (pr.m <= 0 || pr.n <= 0) return 0;
  // The planner's split count first: a plan with one k-split (small k, or
  // k = 0) needs no partials and runs at any size. Otherwise one split's
  // partials are m * n FP64 (complex: pairs); with fewer splits than the
  // planner chose they are made to fit the static array, and problems where
  // not even two fit are refused.
  const size_t per_split = size_t(pr.m) * size_t(pr.n) * (dtype_is_complex(pr.dtype) ? 16 : 8);
  DmmaPlan plan = dmma_plan(pr, num_sms);
  if (plan.workspace_bytes > SPLAB_NOALLOC_SCRATCH_BYTES) {
    const size_t fit = size_t(SPLAB_NOALLOC_SCRATCH_BYTES) / per_split;
    if (fit < 2) return 2;
    plan = dmma_plan(pr, num_sms, int(std::min<size_t>(fit, 4096)));
    if (plan.workspace_bytes > SPLAB_NOALLOC_SCRATCH_BYTES) return 2;
  }
  void* scratch = nullptr;
  if (plan.workspace_bytes > 0 && noalloc_scratch_address(&scratch) != cudaSuccess) return 3;
  return dmma_gemm(pr, plan, scratch, st) == cudaSuccess ? 0 : 3;
}

// ---------------------------------------------------------------------------
// Batched grouped contraction: many independent problems of one dtype and
// operand layout in one persistent launch (plus one grouped reduction),
// captured in a CUDA graph, with the k-chunk size picked by measurement.

// Grouped reduction: blockIdx.y = problem, x covers its elements.
template <int DT>
__global__ void reduce_partials_grouped_kernel(const DmmaParams* __restrict__ params,
                                               const int* __restrict__ splits, int tile_m,
                                               int tile_n) {
  const DmmaParams& p = params[blockIdx.y];
  const int ns = splits[blockIdx.y];
  const int64_t total = p.m * p.n;
  constexpr bool CPLX = dtype_is_complex(DT);
  for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < total;
       idx += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = idx % p.m, j = idx / p.m;
    if (p.fill_mode != 0) {
      const int64_t ti = (i / tile_m) * tile_m, tj = (j / tile_n) * tile_n;
      if (!tile_is_active(p.fill_mode, ti, tj, ::min((int64_t)tile_m, p.m - ti),
                          ::min((int64_t)tile_n, p.n - tj), p.fill_ro, p.fill_co))
        continue;
    }
    double sr = 0.0, si = 0.0;
    if constexpr (CPLX) {
      const double2* q = static_cast<const double2*>(p.P) + idx;
      for (int s = 0; s < ns; ++s) {
        const double2 v = q[s * total];
        sr += v.x;
        si += v.y;
      }
    } else {
      const double* q = static_cast<const double*>(p.P) + idx;
      for (int s = 0; s < ns; ++s) sr += q[s * total];
    }
    store_alpha_beta_impl<DT>(p.C, i + j * p.ldc, sr, si, p.alpha_r, p.alpha_i, p.beta_r,
                              p.beta_i);
  }
}

namespace {

template <class Cfg>
int grouped_occupancy() {
  static int occ = -1;
  set_dynamic_smem(reinterpret_cast<const void*>(dmma_gemm_grouped_kernel<Cfg>),
                   Cfg::SMEM_BYTES);
  if (occ < 0) {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, dmma_gemm_grouped_kernel<Cfg>,
                                                      Cfg::THREADS, Cfg::SMEM_BYTES) !=
            cudaSuccess ||
        o < 1)
      o = 1;
    occ = o;
  }
  return occ;
}

}  // namespace

struct BatchPlanImpl {
  int dtype = 0, opA = 0, opB = 0, count = 0;
  int bm = 0, bn = 0, bk = 0;
  std::vector<GemmProblem> probs;
  int64_t kc = 0;  // k per split (multiple of BK)
  int variant = 0;  // tile configuration: 0 default, 1 larger tiles
  std::vector<int64_t> candidates;
  bool tuned = false;
  // one entry per measured (tile configuration, k-chunk)
  std::vector<double> tuning_ms;
  std::vector<int64_t> entry_kc;
  std::vector<int> entry_bm, entry_bn;
  // device-side tables (allocated by the caller's workspace)
  size_t off_params = 0, off_items = 0, off_splits = 0, off_partials = 0, total = 0;
  int n_items = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void* graph_ws = nullptr;
  void* tables_ws = nullptr;  // workspace holding the tables of the chosen configuration
  // private stream the graph is captured on and replayed on (the caller's
  // stream may be the legacy default stream, which cannot be captured)
  cudaStream_t own = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
};

namespace {

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// Work items of the batch for tiles bm x bn and k-chunk kc.
size_t batch_items(const BatchPlanImpl& b, int bm, int bn, int64_t kc) {
  size_t items = 0;
  for (auto& p : b.probs) {
    const int64_t sp = std::max<int64_t>(1, (p.k + kc - 1) / kc);
    items += size_t(sp) * ((p.m + bm - 1) / bm) * ((p.n + bn - 1) / bn);
  }
  return items;
}

// min_bm x min_bn: the smallest tile of the configurations the plan may use
// (sizes the item table)
template <class Cfg>
void batch_geometry(BatchPlanImpl& b, int min_bm, int min_bn) {
  b.bm = Cfg::BM;
  b.bn = Cfg::BN;
  b.bk = Cfg::BK;
  int64_t kmin = INT64_MAX, kmax = 0;
  for (auto& p : b.probs) {
    kmin = std::min<int64_t>(kmin, p.k);
    kmax = std::max<int64_t>(kmax, p.k);
  }
  // candidate k-chunks: powers of two from the one giving at most 24 splits
  // of the longest problem (bounds the partials' memory) up to the smallest
  // k / 2, so that every problem has at least two splits while tuning (the
  // tuning runs write partials only, never C)
  b.candidates.clear();
  int64_t c0 = 16 * Cfg::BK;
  while (c0 * 24 < kmax) c0 *= 2;
  for (int64_t c = c0; c <= std::max<int64_t>(c0, kmin / 2); c *= 2) b.candidates.push_back(c);
  // workspace: tables + partials for the smallest candidate (most splits)
  const int64_t cmin = b.candidates.front();
  size_t partial_bytes = 0;
  const size_t esz = Cfg::CPLX ? 16 : 8;
  for (auto& p : b.probs) {
    const int64_t sp = std::max<int64_t>(1, (p.k + cmin - 1) / cmin);
    partial_bytes += al256(size_t(sp) * p.m * p.n * esz);
  }
  const size_t items = batch_items(b, min_bm, min_bn, cmin);
  b.off_params = 0;
  b.off_splits = al256(sizeof(DmmaParams) * b.count);
  b.off_items = b.off_splits + al256(sizeof(int) * b.count);
  b.off_partials = b.off_items + al256(sizeof(int4) * items);
  b.total = b.off_partials + partial_bytes;
}

// Build the parameter and item tables for k-chunk kc and upload them.
template <class Cfg>
cudaError_t batch_tables(BatchPlanImpl& b, int64_t kc, char* ws, cudaStream_t st) {
  std::vector<DmmaParams> prm(b.count);
  std::vector<int> splits(b.count);
  std::vector<std::pair<int64_t, int4>> items;
  size_t poff = b.off_partials;
  const size_t esz = Cfg::CPLX ? 16 : 8;
  for (int i = 0; i < b.count; ++i) {
    const GemmProblem& pr = b.probs[i];
    DmmaParams p{};
    p.A = pr.A;
    p.B = pr.B;
    p.C = pr.C;
    p.lda = pr.lda;
    p.ldb = pr.ldb;
    p.ldc = pr.ldc;
    p.m = pr.m;
    p.n = pr.n;
    p.k = pr.k;
    const int sp = int(std::max<int64_t>(1, (pr.k + kc - 1) / kc));
    p.k_per_split = kc;
    p.alpha_r = pr.alpha[0];
    p.alpha_i = pr.alpha[1];
    p.beta_r = pr.beta[0];
    p.beta_i = pr.beta[1];
    p.conj_a = pr.opA == 2;
    p.conj_b = pr.opB == 2;
    p.partial = 1;
    p.fill_mode = pr.fill_mode;
    p.fill_ro = pr.fill_ro;
    p.fill_co = pr.fill_co;
    p.P = ws + poff;
    poff += al256(size_t(sp) * pr.m * pr.n * esz);
    prm[i] = p;
    splits[i] = sp;
    const int64_t tiles = ((pr.m + Cfg::BM - 1) / Cfg::BM) * ((pr.n + Cfg::BN - 1) / Cfg::BN);
    for (int s = 0; s < sp; ++s) {
      const int64_t klen = std::min<int64_t>(kc, pr.k - int64_t(s) * kc);
      for (int64_t t = 0; t < tiles; ++t)
        items.push_back({klen, make_int4(i, int(t), s, 0)});
    }
  }
  if (poff > b.total) return cudaErrorInvalidValue;
  // longest items first so the persistent CTAs finish together
  std::stable_sort(items.begin(), items.end(),
                   [](const auto& a, const auto& c) { return a.first > c.first; });
  std::vector<int4> flat(items.size());
  for (size_t i = 0; i < items.size(); ++i) flat[i] = items[i].second;
  b.n_items = int(flat.size());
  cudaError_t e;
  if ((e = cudaMemcpyAsync(ws + b.off_params, prm.data(), sizeof(DmmaParams) * b.count,
                           cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(ws + b.off_splits, splits.data(), sizeof(int) * b.count,
                           cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return e;
  if ((e = cudaMemcpyAsync(ws + b.off_items, flat.data(), sizeof(int4) * flat.size(),
                           cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return e;
  return cudaStreamSynchronize(st);  // host tables go out of scope
}

template <class Cfg>
cudaError_t batch_launch_gemm(BatchPlanImpl& b, char* ws, cudaStream_t st) {
  const int slots = grouped_occupancy<Cfg>() * [] {
    int dev = 0, v = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
  }();
  const int grid = std::max(1, std::min(b.n_items, slots));
  dmma_gemm_grouped_kernel<Cfg><<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, st>>>(
      reinterpret_cast<const DmmaParams*>(ws + b.off_params),
      reinterpret_cast<const int4*>(ws + b.off_items), b.n_items);
  return cudaGetLastError();
}

template <class Cfg>
cudaError_t batch_launch_reduce(BatchPlanImpl& b, char* ws, cudaStream_t st) {
  int64_t maxel = 0;
  for (auto& p : b.probs) maxel = std::max<int64_t>(maxel, p.m * p.n);
  const int threads = 256;
  const unsigned bx = unsigned(std::min<int64_t>((maxel + threads - 1) / threads, 256));
  reduce_partials_grouped_kernel<Cfg::DT><<<dim3(bx, unsigned(b.count)), threads, 0, st>>>(
      reinterpret_cast<const DmmaParams*>(ws + b.off_params),
      reinterpret_cast<const int*>(ws + b.off_splits), Cfg::BM, Cfg::BN);
  return cudaGetLastError();
}

// Time one launch of the grouped GEMM for configuration Cfg and k-chunk kc
// (tables uploaded for it first; a warm-up launch before the timed one).
template <class Cfg>
cudaError_t batch_time(BatchPlanImpl& b, int64_t kc, char* ws, cudaStream_t st, float* ms) {
  cudaError_t e;
  if ((e = batch_tables<Cfg>(b, kc, ws, st)) != cudaSuccess) return e;
  if ((e = batch_launch_gemm<Cfg>(b, ws, st)) != cudaSuccess) return e;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  e = batch_launch_gemm<Cfg>(b, ws, st);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  *ms = 0.f;
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return e;
}

template <class Cfg>
cudaError_t batch_run_cfg(BatchPlanImpl& b, char* ws, cudaStream_t st) {
  cudaError_t e;
  // capture once per workspace on the plan's own stream, then replay there,
  // ordered after / before the caller's stream with events
  if (!b.own) {
    if ((e = cudaStreamCreateWithFlags(&b.own, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&b.ev_in, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&b.ev_out, cudaEventDisableTiming)) != cudaSuccess) return e;
  }
  if (b.tables_ws != ws) {  // a different workspace than the one tuned on
    if ((e = batch_tables<Cfg>(b, b.kc, ws, st)) != cudaSuccess) return e;
    b.tables_ws = ws;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;  // tables uploaded on st
  if (!b.exec || b.graph_ws != ws) {
    if (b.exec) cudaGraphExecDestroy(b.exec);
    if (b.graph) cudaGraphDestroy(b.graph);
    b.exec = nullptr;
    b.graph = nullptr;
    if ((e = cudaStreamBeginCapture(b.own, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return e;
    cudaError_t e1 = batch_launch_gemm<Cfg>(b, ws, b.own);
    cudaError_t e2 = batch_launch_reduce<Cfg>(b, ws, b.own);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b.own, &g);
    if (e1 != cudaSuccess) return e1;
    if (e2 != cudaSuccess) return e2;
    if (e != cudaSuccess) return e;
    b.graph = g;
    if ((e = cudaGraphInstantiate(&b.exec, g, 0)) != cudaSuccess) return e;
    b.graph_ws = ws;
  }
  if ((e = cudaEventRecord(b.ev_in, st)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(b.own, b.ev_in, 0)) != cudaSuccess) return e;
  if ((e = cudaGraphLaunch(b.exec, b.own)) != cudaSuccess) return e;
  if ((e = cudaEventRecord(b.ev_out, b.own)) != cudaSuccess) return e;
  return cudaStreamWaitEvent(st, b.ev_out, 0);
}

template <int DT, int V, class F>
auto with_cfg_v(const GemmProblem& pr, F&& f) {
  if constexpr (V == 0) {
    return with_cfg<DT>(pr, f);
  } else {
    const bool ak = pr.opA != 0, bk = pr.opB == 0;
    if (ak && bk) return f(typename CfgWide<DT, true, true>::type{});
    if (ak && !bk) return f(typename CfgWide<DT, true, false>::type{});
    if (!ak && bk) return f(typename CfgWide<DT, false, true>::type{});
    return f(typename CfgWide<DT, false, false>::type{});
  }
}

template <int DT, class F>
auto with_variant(const GemmProblem& pr, int v, F&& f) {
  return v == 0 ? with_cfg_v<DT, 0>(pr, f) : with_cfg_v<DT, 1>(pr, f);
}

// Run f with the configuration of the plan's dtype, op pair and tile variant.
template <class F>
auto batch_dispatch(const BatchPlanImpl& b, int variant, F&& f) {
  GemmProblem pr{};
  pr.dtype = b.dtype;
  pr.opA = b.opA;
  pr.opB = b.opB;
  switch (pr.dtype) {
    case kR32: return with_variant<kR32>(pr, variant, f);
    case kR64: return with_variant<kR64>(pr, variant, f);
    case kC32: return with_variant<kC32>(pr, variant, f);
    default: return with_variant<kC64>(pr, variant, f);
  }
}

}  // namespace

BatchPlanImpl* batch_create(int dtype, const std::vector<GemmProblem>& probs) {
  auto* b = new BatchPlanImpl();
  b->dtype = dtype;
  b->opA = probs.front().opA;
  b->opB = probs.front().opB;
  b->count = int(probs.size());
  b->probs = probs;
  int min_bm = 1 << 30, min_bn = 1 << 30;
  for (int v = 0; v < kBatchTileVariants; ++v)
    batch_dispatch(*b, v, [&](auto cfg) {
      min_bm = std::min(min_bm, decltype(cfg)::BM);
      min_bn = std::min(min_bn, decltype(cfg)::BN);
      return 0;
    });
  batch_dispatch(*b, 0, [&](auto cfg) {
    batch_geometry<decltype(cfg)>(*b, min_bm, min_bn);
    return 0;
  });
  return b;
}

size_t batch_workspace(const BatchPlanImpl* b) { return b->total; }

cudaError_t batch_run(BatchPlanImpl* b, void* ws, cudaStream_t st, bool autotune) {
  char* w = static_cast<char*>(ws);
  cudaError_t e;
  if (!b->tuned) {
    b->tuning_ms.clear();
    b->entry_kc.clear();
    b->entry_bm.clear();
    b->entry_bn.clear();
    if (autotune) {
      // measure every (tile configuration, k-chunk) pair and keep the fastest
      double best = 1e30;
      for (int v = 0; v < kBatchTileVariants; ++v)
        for (int64_t kc : b->candidates) {
          float ms = 0.f;
          e = batch_dispatch(*b, v, [&](auto cfg) {
            b->entry_bm.push_back(decltype(cfg)::BM);
            b->entry_bn.push_back(decltype(cfg)::BN);
            return batch_time<decltype(cfg)>(*b, kc, w, st, &ms);
          });
          if (e != cudaSuccess) return e;
          b->tuning_ms.push_back(ms);
          b->entry_kc.push_back(kc);
          if (ms < best) {
            best = ms;
            b->variant = v;
            b->kc = kc;
          }
        }
    } else {
      // model choice: default tiles, the third candidate (8 or more k-tiles
      // per split and several splits per problem for these sizes)
      b->variant = 0;
      b->kc = b->candidates.size() > 2 ? b->candidates[2] : b->candidates.back();
    }
    e = batch_dispatch(*b, b->variant, [&](auto cfg) {
      b->bm = decltype(cfg)::BM;
      b->bn = decltype(cfg)::BN;
      return batch_tables<decltype(cfg)>(*b, b->kc, w, st);
    });
    if (e != cudaSuccess) return e;
    b->tables_ws = ws;
    b->tuned = true;
  }
  return batch_dispatch(*b, b->variant,
                        [&](auto cfg) { return batch_run_cfg<decltype(cfg)>(*b, w, st); });
}

void batch_destroy(BatchPlanImpl* b) {
  if (!b) return;
  if (b->own) cudaStreamSynchronize(b->own);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->ev_in) cudaEventDestroy(b->ev_in);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
}

int64_t batch_kc(const BatchPlanImpl* b) { return b->kc; }
const std::vector<double>& batch_tuning(const BatchPlanImpl* b) { return b->tuning_ms; }
const std::vector<int64_t>& batch_candidates(const BatchPlanImpl* b) {
  return b->tuned && !b->entry_kc.empty() ? b->entry_kc : b->candidates;
}
void batch_tiles(const BatchPlanImpl* b, int* bm, int* bn, std::vector<int>* entry_bm,
                 std::vector<int>* entry_bn) {
  *bm = b->bm;
  *bn = b->bn;
  *entry_bm = b->entry_bm;
  *entry_bn = b->entry_bn;
}
}  // namespace splab
