// splab_* C ABI: argument checks and dispatch to the sm_100a kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>
#include <type_traits>
#include <utility>

#include "../../../include/splab.h"
#include "common.cuh"
#include "gemm_dmma.cuh"
#include "ozaki.cuh"
#include "tf32x3.cuh"
#include "batch_seq.cuh"

namespace splab {

PhaseEvents& phase_events() {
  static thread_local PhaseEvents pe;
  return pe;
}

cudaError_t set_dynamic_smem(const void* func, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, func})) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.insert({dev, func});
  return e;
}

namespace {

int num_sms() {
  int dev = 0;
  cudaGetDevice(&dev);
  static int cached[64] = {0};
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1)
      v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}

bool valid_problem(int dtype, int opA, int opB, int64_t m, int64_t n, int64_t k, int64_t lda,
                   int64_t ldb, int64_t ldc) {
  if (dtype < 0 || dtype > 3) return false;
  if (opA < 0 || opA > 2 || opB < 0 || opB > 2) return false;
  if (m < 0 || n < 0 || k < 0) return false;
  if (lda < std::max<int64_t>(1, opA == 0 ? m : k)) return false;
  if (ldb < std::max<int64_t>(1, opB == 0 ? k : n)) return false;
  if (ldc < std::max<int64_t>(1, m)) return false;
  return true;
}

GemmProblem make_problem(int dtype, int opA, int opB, int64_t m, int64_t n, int64_t k,
                         const void* alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
                         const void* beta, void* C, int64_t ldc, int fill, int64_t ro,
                         int64_t co) {
  GemmProblem p{};
  p.dtype = dtype;
  p.opA = opA;
  p.opB = opB;
  p.m = m;
  p.n = n;
  p.k = k;
  p.A = A;
  p.lda = lda;
  p.B = B;
  p.ldb = ldb;
  p.C = C;
  p.ldc = ldc;
  p.fill_mode = fill;
  p.fill_ro = ro;
  p.fill_co = co;
  const bool dbl = dtype_is_double(dtype), cplx = dtype_is_complex(dtype);
  for (int i = 0; i < 2; ++i) {
    p.alpha[i] = p.beta[i] = 0.0;
    if (i == 1 && !cplx) break;
    p.alpha[i] = dbl ? static_cast<const double*>(alpha)[i] : static_cast<const float*>(alpha)[i];
    p.beta[i] = dbl ? static_cast<const double*>(beta)[i] : static_cast<const float*>(beta)[i];
  }
  return p;
}

// Path selection. An explicit path is taken when it supports the problem
// (Ozaki: every op pair whose in-place operands fit its slicer's grid;
// 3xTF32: float dtypes only), else the FP64 DMMA kernel runs. AUTO takes the path with the least
// modelled time among the supported ones whose workspace fits in a quarter of
// the device memory. The model's constants were measured on B200 (complex and
// real, m = n from 128 to 2048, k from 8192 to 65536, and the k = 250000
// configurations): DMMA at 33 / 29 TFLOP/s (complex / real) plus 0.05 ms; the
// Ozaki path as slicing (6.0e-13 s per real element and modulus, plus the
// norms' read at 6 TB/s, which rows of 131072 reals or more mostly skip: a
// 1/16 sample), INT8 GEMM at 2.8 POP/s scaled by how evenly its work
// units fill the 74 CTA pairs, reconstruction (3e-12 s per real output and
// modulus) and 0.08 ms; 3xTF32 as splitting (bytes at 5.5 TB/s), three TF32
// products at 480 TFLOP/s scaled by the same fill, and 0.05 ms. The choice only
// depends on the problem and the device (no free-memory query), so that
// resolving a path, sizing its workspace and running it agree.
namespace model {

constexpr int kPairs = 74;

double fill(double units) {
  if (units <= 0) return 1.0;
  const double rounds = std::ceil(units / kPairs);
  return units / (rounds * kPairs);
}

double dmma_ms(const GemmProblem& p) {
  const bool c = dtype_is_complex(p.dtype);
  const double flops = double(p.m) * p.n * p.k * (c ? 8.0 : 2.0);
  return flops / (c ? 33e12 : 29e12) * 1e3 + 0.05;
}

double ozaki_ms(const GemmProblem& p) {
  const bool c = dtype_is_complex(p.dtype);
  const int nmod = dtype_is_double(p.dtype) ? 15 : 9;
  const double nsub = c ? 3.0 : 1.0;  // complex: three real products per modulus
  const double K2 = c ? 2.0 * p.k : double(p.k);
  const double kp = std::ceil(p.k / 128.0) * 128.0;
  const double reals = double(p.m + p.n) * K2;
  // per real element and modulus: complex rows feed three residue planes
  // norms: one read per operand; a k-major one with rows of 131072 reals or
  // more only reads a 1/16 sample (one-pass scaling)
  const double esz = dtype_is_double(p.dtype) ? 8 : 4;
  auto norm_rows = [&](double rows, bool k_major) {
    return rows * K2 * esz / 6e12 / (k_major && K2 >= 131072 ? 16.0 : 1.0);
  };
  const double slice = (c ? 6.0e-13 : 4.0e-13) * reals * nmod +
                       norm_rows(p.m, !(p.opA == 0 && !ozaki_copies_a(p))) +
                       norm_rows(p.n, p.opB == 0);
  const double tiles = std::ceil(p.m / 256.0) * std::ceil(p.n / 256.0) * nsub;
  const double chunks = std::ceil(kp / 128.0 / 976.0);
  const double gemm = 2.0 * nmod * nsub * p.m * p.n * kp / (2.8e15 * fill(nmod * chunks * tiles));
  const double recon = (c ? 3e-12 * 2.0 : 2e-12) * p.m * double(p.n) * nmod;
  // op(A) = N beyond the in-place reach: A is first copied k-major (one read,
  // one write)
  const double transpose =
      ozaki_copies_a(p) ? 2.0 * p.m * K2 * (dtype_is_double(p.dtype) ? 8 : 4) / 6e12 : 0.0;
  return (slice + gemm + recon + transpose) * 1e3 + 0.08;
}

double tf32x3_ms(const GemmProblem& p) {
  const bool c = dtype_is_complex(p.dtype);
  const double K2 = c ? 2.0 * p.k : double(p.k), nb = c ? 2.0 * p.n : double(p.n);
  const double kp = std::ceil(K2 / 32.0) * 32.0;
  const double bytes = double(p.m + p.n) * K2 * 4 + (p.m + nb) * kp * 8;
  const double tiles = std::ceil(p.m / 256.0) * std::ceil(nb / 128.0);
  const double splits = std::max(1.0, std::floor(kp / 32.0 / 64.0));
  // the split count is chosen to balance the units over the pairs when k allows
  const double units = tiles * splits;
  const double gemm = 6.0 * p.m * nb * kp / (4.8e14 * (units >= kPairs ? 0.95 : units / kPairs));
  return (bytes / 5.5e12 + gemm) * 1e3 + 0.05;
}

}  // namespace model

size_t device_total_memory() {
  static size_t total = 0;
  if (!total) {
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    total = t;
  }
  return total;
}

// Operand normalisation for the tensor-core paths, whose kernels contract
// k-major operands (op(B) = N; on 3xTF32 also op(A) in {T, C}): op(B) in
// {T, C} is first copied k-major (conjugated for C) into the head of the
// workspace, and on 3xTF32 so is A when op(A) = N. The path then runs on the
// normalised problem with the rest of the workspace. The local gemm() takes
// every op pair (reference include/spla/gemm.hpp:66-97,
// src/gemm/gemm_gpu.cpp:59-174).
struct Normalized {
  GemmProblem p;  // the problem the path runs (pointers to the copies set at run time)
  bool copyA = false, copyB = false;
  int64_t ldAn = 0, ldBn = 0;
  size_t offA = 0, offB = 0, prefix = 0;  // byte offsets of the copies; the path's workspace
};

size_t align_up256(size_t x) { return (x + 255) & ~size_t(255); }

Normalized normalize(const GemmProblem& p, int rp) {
  Normalized N;
  N.p = p;
  if (rp != SPLAB_PATH_OZAKI && rp != SPLAB_PATH_TF32X3) return N;
  const size_t esz = size_t(dtype_bytes(p.dtype));
  const int64_t kn = (std::max<int64_t>(p.k, 1) + 7) / 8 * 8;  // 16-byte aligned rows
  size_t off = 0;
  if (p.opB != 0 && rp == SPLAB_PATH_TF32X3) {  // the Ozaki path reads op(B) = T, C in place
    N.copyB = true;
    N.ldBn = kn;
    N.offB = off;
    off = align_up256(off + esz * size_t(p.n) * size_t(kn));
    N.p.opB = 0;
    N.p.ldb = kn;
  }
  if (rp == SPLAB_PATH_TF32X3 && p.opA == 0) {
    N.copyA = true;
    N.ldAn = kn;
    N.offA = off;
    off = align_up256(off + esz * size_t(p.m) * size_t(kn));
    N.p.opA = 1;
    N.p.lda = kn;
  }
  N.prefix = off;
  return N;
}

// The k-major view a tensor-core path would run (for support checks).
GemmProblem k_major_view(const GemmProblem& p, bool copy_a) {
  GemmProblem q = p;
  q.opB = 0;
  if (copy_a && q.opA == 0) q.opA = 1;
  return q;
}

// Y (k x rows, column-major, ldy) <- X (rows x k, column-major, ldx),
// conjugated when `conj` (complex element types): a 32 x 32 tile through
// shared memory, reads coalesced along rows, writes along k.
template <typename E>
__global__ void to_k_major(const E* __restrict__ X, int64_t ldx, int64_t rows, int64_t k,
                           int conj, E* __restrict__ Y, int64_t ldy) {
  __shared__ E tile[32][33];
  const int64_t r0 = int64_t(blockIdx.x) * 32;
  for (int64_t k0 = int64_t(blockIdx.y) * 32; k0 < k; k0 += int64_t(gridDim.y) * 32) {
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
      const int64_t r = r0 + threadIdx.x, kk = k0 + j;
      if (r < rows && kk < k) tile[j][threadIdx.x] = X[r + kk * ldx];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
      const int64_t r = r0 + j, kk = k0 + threadIdx.x;
      if (r < rows && kk < k) {
        E v = tile[threadIdx.x][j];
        if constexpr (sizeof(E) == 8 && !std::is_same<E, double>::value) {
          if (conj) v.y = -v.y;
        } else if constexpr (sizeof(E) == 16) {
          if (conj) v.y = -v.y;
        }
        Y[kk + r * ldy] = v;
      }
    }
    __syncthreads();
  }
}

cudaError_t launch_to_k_major(int dtype, const void* X, int64_t ldx, int64_t rows, int64_t k,
                              bool conj, void* Y, int64_t ldy, cudaStream_t st) {
  if (rows <= 0 || k <= 0) return cudaSuccess;
  const dim3 block(32, 8);
  const dim3 grid(unsigned((rows + 31) / 32), unsigned(std::min<int64_t>((k + 31) / 32, 65535)));
  auto go = [&](auto tag) {
    using E = decltype(tag);
    to_k_major<E><<<grid, block, 0, st>>>(static_cast<const E*>(X), ldx, rows, k, conj ? 1 : 0,
                                          static_cast<E*>(Y), ldy);
  };
  switch (dtype) {
    case kR32: go(float{}); break;
    case kR64: go(double{}); break;
    case kC32: go(float2{}); break;
    default: go(double2{}); break;
  }
  return cudaGetLastError();
}

// The copies of a normalised problem, on `st`; redirects N.p's operands.
cudaError_t run_normalization(Normalized& N, const GemmProblem& p, char* ws, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  if (N.copyB) {
    // op(B) is k x n: B holds n x k (column-major, ldb)
    e = launch_to_k_major(p.dtype, p.B, p.ldb, p.n, p.k, p.opB == 2, ws + N.offB, N.ldBn, st);
    if (e != cudaSuccess) return e;
    N.p.B = ws + N.offB;
  }
  if (N.copyA) {
    e = launch_to_k_major(p.dtype, p.A, p.lda, p.m, p.k, false, ws + N.offA, N.ldAn, st);
    if (e != cudaSuccess) return e;
    N.p.A = ws + N.offA;
  }
  return e;
}

size_t path_workspace(const GemmProblem& p, int rp, int moduli) {
  if (rp == SPLAB_PATH_TF32X3 || rp == SPLAB_PATH_OZAKI) {
    const Normalized N = normalize(p, rp);
    return N.prefix + (rp == SPLAB_PATH_TF32X3 ? tf32x3_workspace_bytes(N.p)
                                               : ozaki_workspace_bytes(N.p, moduli));
  }
  return dmma_plan(p, num_sms()).workspace_bytes;
}

int resolve_path(const GemmProblem& p, int path, int moduli) {
  const bool oz = ozaki_supported(p);  // op(B) = T, C read in place by the path itself
  const bool tf = tf32x3_supported(k_major_view(p, true));
  if (path == SPLAB_PATH_TF32X3) return tf ? SPLAB_PATH_TF32X3 : SPLAB_PATH_DMMA;
  if (path == SPLAB_PATH_OZAKI) return oz ? SPLAB_PATH_OZAKI : SPLAB_PATH_DMMA;
  if (path == SPLAB_PATH_DMMA || p.m <= 0 || p.n <= 0 || p.k <= 0) return SPLAB_PATH_DMMA;
  const size_t cap = device_total_memory() / 4;
  // the k-major copies of a normalised problem: one read and one write each
  const double esz = dtype_bytes(p.dtype);
  const double copyB = p.opB != 0 ? 2.0 * p.n * p.k * esz / 6e12 * 1e3 : 0.0;
  const double copyA = p.opA == 0 ? 2.0 * p.m * p.k * esz / 6e12 * 1e3 : 0.0;
  int best = SPLAB_PATH_DMMA;
  double best_ms = model::dmma_ms(p);
  if (oz && path_workspace(p, SPLAB_PATH_OZAKI, moduli) <= cap) {
    const double t = model::ozaki_ms(k_major_view(p, false));
    if (t < 0.9 * best_ms) {
      best = SPLAB_PATH_OZAKI;
      best_ms = t;
    }
  }
  if (tf && path_workspace(p, SPLAB_PATH_TF32X3, moduli) <= cap) {
    const double t = model::tf32x3_ms(k_major_view(p, true)) + copyB + copyA;
    if (t < 0.9 * best_ms) best = SPLAB_PATH_TF32X3;
  }
  return best;
}

__global__ void block_cyclic_info_kernel(int64_t rb, int64_t cb, int64_t gr, int64_t gc,
                                         int64_t nr, int64_t nc, int64_t ro, int64_t co,
                                         const int64_t* __restrict__ ids, int64_t count,
                                         int64_t* __restrict__ out) {
  const int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (t >= count) return;
  const int64_t firstRow = (ro / rb) * rb, firstCol = (co / cb) * cb;
  const int64_t numBlockRows = (ro - firstRow + nr + rb - 1) / rb;
  const int64_t b = ids[t];
  const int64_t bRow = b % numBlockRows, bCol = b / numBlockRows;
  const int64_t gbRow = bRow + ro / rb, gbCol = bCol + co / cb;
  const int64_t gRow = max(ro, firstRow + bRow * rb), gCol = max(co, firstCol + bCol * cb);
  const int64_t endRow = min((gbRow + 1) * rb, ro + nr), endCol = min((gbCol + 1) * cb, co + nc);
  int64_t* o = out + 9 * t;
  o[0] = gRow;
  o[1] = gCol;
  o[2] = gRow - ro;
  o[3] = gCol - co;
  o[4] = (gbRow / gr) * rb + gRow % rb;
  o[5] = (gbCol / gc) * cb + gCol % cb;
  o[6] = endRow - gRow;
  o[7] = endCol - gCol;
  o[8] = (gbRow % gr) + (gbCol % gc) * gr;
}

// Block copies of the distributed exchange: for every block descriptor
// (srcOff, srcLd, dstOff, dstLd, rows, cols) in elements,
// dst[dstOff + i + j dstLd] = alpha src[srcOff + i + j srcLd] + beta dst[...]
// (dst not read when beta = 0). blockIdx.y walks the blocks, blockIdx.x and
// the threads their elements.
template <typename T, bool CPLX>
__global__ void copy_blocks_kernel(const T* __restrict__ src, T* __restrict__ dst,
                                   const int64_t* __restrict__ desc, int64_t count, double ar,
                                   double ai, double br, double bi) {
  for (int64_t b = blockIdx.y; b < count; b += gridDim.y) {
    const int64_t* d = desc + 6 * b;
    const int64_t so = d[0], sld = d[1], dof = d[2], dld = d[3], rows = d[4], cols = d[5];
    const int64_t total = rows * cols;
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
         e += int64_t(gridDim.x) * blockDim.x) {
      const int64_t i = e % rows, j = e / rows;
      const int64_t s = so + i + j * sld, t = dof + i + j * dld;
      if (CPLX) {
        const double xr = double(src[2 * s]), xi = double(src[2 * s + 1]);
        double yr = ar * xr - ai * xi, yi = ar * xi + ai * xr;
        if (br != 0.0 || bi != 0.0) {
          const double cr = double(dst[2 * t]), ci = double(dst[2 * t + 1]);
          yr += br * cr - bi * ci;
          yi += br * ci + bi * cr;
        }
        dst[2 * t] = T(yr);
        dst[2 * t + 1] = T(yi);
      } else {
        double y = ar * double(src[s]);
        if (br != 0.0) y += br * double(dst[t]);
        dst[t] = T(y);
      }
    }
  }
}

// Host form of the block-cyclic map (the device kernel above, one block at a
// time): BlockCyclicGenerator::get_block_info
// (src/block_generation/block_cyclic_generator.cpp:59-100).
void block_cyclic_info_host(int64_t rb, int64_t cb, int64_t gr, int64_t gc, int64_t nr,
                            int64_t nc, int64_t ro, int64_t co, int64_t b, int64_t* o) {
  const int64_t firstRow = (ro / rb) * rb, firstCol = (co / cb) * cb;
  const int64_t numBlockRows = (ro - firstRow + nr + rb - 1) / rb;
  const int64_t bRow = b % numBlockRows, bCol = b / numBlockRows;
  const int64_t gbRow = bRow + ro / rb, gbCol = bCol + co / cb;
  const int64_t gRow = std::max(ro, firstRow + bRow * rb), gCol = std::max(co, firstCol + bCol * cb);
  const int64_t endRow = std::min((gbRow + 1) * rb, ro + nr);
  const int64_t endCol = std::min((gbCol + 1) * cb, co + nc);
  o[0] = gRow;
  o[1] = gCol;
  o[2] = gRow - ro;
  o[3] = gCol - co;
  o[4] = (gbRow / gr) * rb + gRow % rb;
  o[5] = (gbCol / gc) * cb + gCol % cb;
  o[6] = endRow - gRow;
  o[7] = endCol - gCol;
  o[8] = (gbRow % gr) + (gbCol % gc) * gr;
}

// A batch plan: the grouped FP64 launch or a tensor-core sequence.
struct BatchHandle {
  BatchPlanImpl* grouped = nullptr;
  SeqBatch* seq = nullptr;
};

}  // namespace
}  // namespace splab

using namespace splab;

extern "C" {

const char* splab_status_string(int status) {
  switch (status) {
    case SPLAB_OK: return "ok";
    case SPLAB_ERR_INVALID: return "invalid argument";
    case SPLAB_ERR_WORKSPACE: return "workspace missing or too small";
    case SPLAB_ERR_LAUNCH: return "CUDA launch or runtime error";
    case SPLAB_ERR_UNSUPPORTED: return "path not supported for this dtype or device";
    case SPLAB_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "unknown status";
  }
}

int splab_gemm_path(int dtype, int path, int opA, int opB, int64_t m, int64_t n, int64_t k) {
  GemmProblem p{};
  p.dtype = dtype;
  p.opA = opA;
  p.opB = opB;
  p.m = m;
  p.n = n;
  p.k = k;
  if (dtype < 0 || dtype > 3 || m <= 0 || n <= 0 || k < 0) return SPLAB_PATH_DMMA;
  return resolve_path(p, path, 0);
}

size_t splab_gemm_workspace_size(int dtype, int path, int opA, int opB, int64_t m, int64_t n,
                                 int64_t k, int ozakiModuli) {
  if (dtype < 0 || dtype > 3 || m <= 0 || n <= 0 || k < 0) return 0;
  GemmProblem p{};
  p.dtype = dtype;
  p.opA = opA;
  p.opB = opB;
  p.m = m;
  p.n = n;
  p.k = k;
  return path_workspace(p, resolve_path(p, path, ozakiModuli), ozakiModuli);
}

int splab_gemm_check(int dtype, int path, int opA, int opB, int64_t m, int64_t n, int64_t k,
                     int ozakiModuli, void* workspace, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GemmProblem p{};
  p.dtype = dtype;
  p.opA = opA;
  p.opB = opB;
  p.m = m;
  p.n = n;
  p.k = k;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SPLAB_ERR_LAUNCH;
  if (m <= 0 || n <= 0 || !workspace) return SPLAB_OK;
  const int rp = resolve_path(p, path, ozakiModuli);
  const Normalized N = normalize(p, rp);
  void* pw = static_cast<char*>(workspace) + N.prefix;
  if (rp == SPLAB_PATH_TF32X3)
    return tf32x3_status(N.p, pw, st) ? SPLAB_ERR_TIMEOUT : SPLAB_OK;
  if (rp != SPLAB_PATH_OZAKI) return SPLAB_OK;
  return ozaki_status(N.p, ozakiModuli, pw, st) ? SPLAB_ERR_TIMEOUT : SPLAB_OK;
}

int splab_gemm(int dtype, int path, int opA, int opB, int64_t m, int64_t n, int64_t k,
               const void* alpha, const void* A, int64_t lda, const void* B, int64_t ldb,
               const void* beta, void* C, int64_t ldc, int fill, int64_t ro, int64_t co,
               int ozakiModuli, void* workspace, size_t workspaceBytes, void* stream) {
  if (!valid_problem(dtype, opA, opB, m, n, k, lda, ldb, ldc)) return SPLAB_ERR_INVALID;
  if (path < 0 || path > 3 || fill < 0 || fill > 2 || !alpha || !beta) return SPLAB_ERR_INVALID;
  if (m == 0 || n == 0) return SPLAB_OK;
  if (!C || (k > 0 && (!A || !B))) return SPLAB_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GemmProblem p = make_problem(dtype, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                               fill, ro, co);
  cudaError_t err;
  if (ozakiModuli != 0 && (ozakiModuli < 8 || ozakiModuli > 16)) return SPLAB_ERR_INVALID;
  const int rp = resolve_path(p, path, ozakiModuli);
  if (rp == SPLAB_PATH_TF32X3 || rp == SPLAB_PATH_OZAKI) {
    const size_t need = path_workspace(p, rp, ozakiModuli);
    if (need > workspaceBytes || (need && !workspace)) return SPLAB_ERR_WORKSPACE;
    Normalized N = normalize(p, rp);
    char* ws = static_cast<char*>(workspace);
    err = run_normalization(N, p, ws, st);
    if (err == cudaSuccess)
      err = rp == SPLAB_PATH_TF32X3
                ? tf32x3_gemm(N.p, ws + N.prefix, workspaceBytes - N.prefix, st)
                : ozaki_gemm(N.p, ozakiModuli, ws + N.prefix, workspaceBytes - N.prefix, st);
  } else {
    const DmmaPlan plan = dmma_plan(p, num_sms());
    if (plan.workspace_bytes > workspaceBytes || (plan.workspace_bytes && !workspace))
      return SPLAB_ERR_WORKSPACE;
    err = dmma_gemm(p, plan, workspace, st);
  }
  if (err != cudaSuccess && std::getenv("SPLA_B200_DEBUG"))
    std::fprintf(stderr, "splab_gemm: %s (%s) dtype %d path %d m %lld n %lld k %lld\n",
                 cudaGetErrorName(err), cudaGetErrorString(err), dtype, path, (long long)m,
                 (long long)n, (long long)k);
  return err == cudaSuccess ? SPLAB_OK : SPLAB_ERR_LAUNCH;
}

int splab_gemm_dmma_noalloc(int dtype, int opA, int opB, int64_t m, int64_t n, int64_t k,
                            const void* alpha, const void* A, int64_t lda, const void* B,
                            int64_t ldb, const void* beta, void* C, int64_t ldc, int fill,
                            int64_t ro, int64_t co, void* stream) {
  if (!valid_problem(dtype, opA, opB, m, n, k, lda, ldb, ldc)) return SPLAB_ERR_INVALID;
  if (fill < 0 || fill > 2 || !alpha || !beta) return SPLAB_ERR_INVALID;
  if (m == 0 || n == 0) return SPLAB_OK;
  if (!C || (k > 0 && (!A || !B))) return SPLAB_ERR_INVALID;
  GemmProblem p = make_problem(dtype, opA, opB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                               fill, ro, co);
  const int rc = dmma_gemm_noalloc(p, num_sms(), static_cast<cudaStream_t>(stream));
  if (rc == 2) return SPLAB_ERR_WORKSPACE;
  return rc == 0 ? SPLAB_OK : SPLAB_ERR_LAUNCH;
}

int splab_batch_create(int dtype, int count, const splab_problem* problems, void** plan,
                       size_t* workspaceBytes) {
  return splab_batch_create_path(dtype, SPLAB_PATH_DMMA, count, problems, plan, workspaceBytes);
}

int splab_batch_create_path(int dtype, int path, int count, const splab_problem* problems,
                            void** plan, size_t* workspaceBytes) {
  if (dtype < 0 || dtype > 3 || path < 0 || path > 3 || count < 1 || !problems || !plan ||
      !workspaceBytes)
    return SPLAB_ERR_INVALID;
  std::vector<GemmProblem> probs;
  probs.reserve(count);
  for (int i = 0; i < count; ++i) {
    const splab_problem& q = problems[i];
    if (q.opA != problems[0].opA || q.opB != problems[0].opB) return SPLAB_ERR_INVALID;
    if (!valid_problem(dtype, q.opA, q.opB, q.m, q.n, q.k, q.lda, q.ldb, q.ldc))
      return SPLAB_ERR_INVALID;
    if (q.m > 0 && q.n > 0 && (!q.C || (q.k > 0 && (!q.A || !q.B)))) return SPLAB_ERR_INVALID;
    GemmProblem p{};
    p.dtype = dtype;
    p.opA = q.opA;
    p.opB = q.opB;
    p.m = q.m;
    p.n = q.n;
    p.k = q.k;
    p.A = q.A;
    p.lda = q.lda;
    p.B = q.B;
    p.ldb = q.ldb;
    p.C = q.C;
    p.ldc = q.ldc;
    const bool cplx = dtype_is_complex(dtype);
    p.alpha[0] = q.alpha[0];
    p.alpha[1] = cplx ? q.alpha[1] : 0.0;
    p.beta[0] = q.beta[0];
    p.beta[1] = cplx ? q.beta[1] : 0.0;
    if (p.m > 0 && p.n > 0) probs.push_back(p);
  }
  if (probs.empty()) return SPLAB_ERR_INVALID;
  auto* h = new BatchHandle();
  if (path == SPLAB_PATH_OZAKI || path == SPLAB_PATH_TF32X3) {
    h->seq = seq_batch_create(path, probs);
    if (!h->seq) {
      delete h;
      return SPLAB_ERR_UNSUPPORTED;
    }
    *workspaceBytes = seq_batch_workspace(h->seq);
  } else {
    h->grouped = batch_create(dtype, probs);
    *workspaceBytes = batch_workspace(h->grouped);
  }
  *plan = h;
  return SPLAB_OK;
}

int splab_batch_run(void* plan, void* workspace, size_t workspaceBytes, int autotune,
                    void* stream) {
  if (!plan) return SPLAB_ERR_INVALID;
  BatchHandle* h = static_cast<BatchHandle*>(plan);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (h->seq) {
    if (!workspace || workspaceBytes < seq_batch_workspace(h->seq)) return SPLAB_ERR_WORKSPACE;
    e = seq_batch_run(h->seq, workspace, st);
  } else {
    if (!workspace || workspaceBytes < batch_workspace(h->grouped)) return SPLAB_ERR_WORKSPACE;
    e = batch_run(h->grouped, workspace, st, autotune != 0);
  }
  return e == cudaSuccess ? SPLAB_OK : SPLAB_ERR_LAUNCH;
}

int splab_batch_check(void* plan, void* workspace, void* stream) {
  if (!plan) return SPLAB_ERR_INVALID;
  BatchHandle* h = static_cast<BatchHandle*>(plan);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaStreamSynchronize(st) != cudaSuccess) return SPLAB_ERR_LAUNCH;
  if (!h->seq || !workspace) return SPLAB_OK;
  return seq_batch_status(h->seq, workspace, st) ? SPLAB_ERR_TIMEOUT : SPLAB_OK;
}

int splab_batch_info(void* plan, int64_t* kChunk, int* nCandidates, int64_t* candidates,
                     double* tuningMs) {
  if (!plan) return SPLAB_ERR_INVALID;
  const BatchHandle* h = static_cast<const BatchHandle*>(plan);
  if (h->seq) {  // no k-chunk to tune: every instance runs its path's own split
    if (kChunk) *kChunk = 0;
    if (nCandidates) *nCandidates = 0;
    return SPLAB_OK;
  }
  const BatchPlanImpl* b = h->grouped;
  if (kChunk) *kChunk = batch_kc(b);
  const auto& c = batch_candidates(b);
  const auto& t = batch_tuning(b);
  const int nc = int(std::min<size_t>(c.size(), 32));
  if (nCandidates) *nCandidates = nc;
  for (int i = 0; i < nc; ++i) {
    if (candidates) candidates[i] = c[i];
    if (tuningMs) tuningMs[i] = i < int(t.size()) ? t[i] : -1.0;
  }
  return SPLAB_OK;
}

int splab_batch_tiles(void* plan, int* tileM, int* tileN, int* nEntries, int* entryTileM,
                      int* entryTileN) {
  if (!plan) return SPLAB_ERR_INVALID;
  const BatchHandle* h = static_cast<const BatchHandle*>(plan);
  if (h->seq) {  // the tensor-core paths pick their own tiles
    if (tileM) *tileM = 0;
    if (tileN) *tileN = 0;
    if (nEntries) *nEntries = 0;
    return SPLAB_OK;
  }
  int bm = 0, bn = 0;
  std::vector<int> ebm, ebn;
  batch_tiles(h->grouped, &bm, &bn, &ebm, &ebn);
  if (tileM) *tileM = bm;
  if (tileN) *tileN = bn;
  const int ne = int(std::min<size_t>(ebm.size(), 32));
  if (nEntries) *nEntries = ne;
  for (int i = 0; i < ne; ++i) {
    if (entryTileM) entryTileM[i] = ebm[i];
    if (entryTileN) entryTileN[i] = ebn[i];
  }
  return SPLAB_OK;
}

int splab_batch_destroy(void* plan) {
  BatchHandle* h = static_cast<BatchHandle*>(plan);
  if (!h) return SPLAB_OK;
  if (h->seq) seq_batch_destroy(h->seq);
  if (h->grouped) batch_destroy(h->grouped);
  delete h;
  return SPLAB_OK;
}

int splab_set_phase_events(void** events, int count) {
  PhaseEvents& pe = phase_events();
  pe.ev = reinterpret_cast<cudaEvent_t*>(events);
  pe.count = events ? count : 0;
  return SPLAB_OK;
}

int splab_block_cyclic_info(int64_t rowsInBlock, int64_t colsInBlock, int64_t gridRows,
                            int64_t gridCols, int64_t globalRows, int64_t globalCols,
                            int64_t rowOffset, int64_t colOffset, const int64_t* blockIdx,
                            int64_t count, int64_t* out, void* stream) {
  if (rowsInBlock < 1 || colsInBlock < 1 || gridRows < 1 || gridCols < 1 || globalRows < 0 ||
      globalCols < 0 || rowOffset < 0 || colOffset < 0 || count < 0)
    return SPLAB_ERR_INVALID;
  if (count == 0) return SPLAB_OK;
  if (!blockIdx || !out) return SPLAB_ERR_INVALID;
  const int threads = 256;
  const int64_t blocks = (count + threads - 1) / threads;
  block_cyclic_info_kernel<<<unsigned(blocks), threads, 0, static_cast<cudaStream_t>(stream)>>>(
      rowsInBlock, colsInBlock, gridRows, gridCols, globalRows, globalCols, rowOffset, colOffset,
      blockIdx, count, out);
  return cudaGetLastError() == cudaSuccess ? SPLAB_OK : SPLAB_ERR_LAUNCH;
}

int64_t splab_block_cyclic_blocks(int64_t rowsInBlock, int64_t colsInBlock, int64_t gridRows,
                                  int64_t gridCols, int64_t globalRows, int64_t globalCols,
                                  int64_t rowOffset, int64_t colOffset, int64_t* out) {
  if (rowsInBlock < 1 || colsInBlock < 1 || gridRows < 1 || gridCols < 1 || globalRows < 0 ||
      globalCols < 0 || rowOffset < 0 || colOffset < 0)
    return -1;
  if (globalRows == 0 || globalCols == 0) return 0;
  const int64_t firstRow = (rowOffset / rowsInBlock) * rowsInBlock;
  const int64_t firstCol = (colOffset / colsInBlock) * colsInBlock;
  const int64_t nbr = (rowOffset - firstRow + globalRows + rowsInBlock - 1) / rowsInBlock;
  const int64_t nbc = (colOffset - firstCol + globalCols + colsInBlock - 1) / colsInBlock;
  const int64_t count = nbr * nbc;
  if (out)
    for (int64_t b = 0; b < count; ++b)
      block_cyclic_info_host(rowsInBlock, colsInBlock, gridRows, gridCols, globalRows, globalCols,
                             rowOffset, colOffset, b, out + 9 * b);
  return count;
}

int splab_copy_blocks(int dtype, const void* src, void* dst, const int64_t* desc, int64_t count,
                      int64_t maxBlockElems, const void* alpha, const void* beta, void* stream) {
  if (dtype < 0 || dtype > 3 || count < 0 || maxBlockElems < 0 || !alpha || !beta)
    return SPLAB_ERR_INVALID;
  if (count == 0 || maxBlockElems == 0) return SPLAB_OK;
  if (!src || !dst || !desc) return SPLAB_ERR_INVALID;
  // all three are dereferenced by the kernel: memory the device cannot reach
  // (pageable host memory) is refused here instead of faulting there
  for (const void* ptr : {src, static_cast<const void*>(dst), static_cast<const void*>(desc)}) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
      cudaGetLastError();
      return SPLAB_ERR_INVALID;
    }
    if (at.type == cudaMemoryTypeUnregistered || at.devicePointer == nullptr)
      return SPLAB_ERR_INVALID;
  }
  const bool dbl = dtype_is_double(dtype), cplx = dtype_is_complex(dtype);
  double a[2] = {0, 0}, b[2] = {0, 0};
  for (int i = 0; i < (cplx ? 2 : 1); ++i) {
    a[i] = dbl ? static_cast<const double*>(alpha)[i] : static_cast<const float*>(alpha)[i];
    b[i] = dbl ? static_cast<const double*>(beta)[i] : static_cast<const float*>(beta)[i];
  }
  const int threads = 256;
  const dim3 grid(unsigned(std::min<int64_t>((maxBlockElems + threads - 1) / threads, 1024)),
                  unsigned(std::min<int64_t>(count, 65535)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  auto go = [&](auto tag, auto cflag) {
    using T = decltype(tag);
    copy_blocks_kernel<T, decltype(cflag)::value><<<grid, threads, 0, st>>>(
        static_cast<const T*>(src), static_cast<T*>(dst), desc, count, a[0], a[1], b[0], b[1]);
  };
  switch (dtype) {
    case kR32: go(float{}, std::false_type{}); break;
    case kR64: go(double{}, std::false_type{}); break;
    case kC32: go(float{}, std::true_type{}); break;
    default: go(double{}, std::true_type{}); break;
  }
  return cudaGetLastError() == cudaSuccess ? SPLAB_OK : SPLAB_ERR_LAUNCH;
}

}  // extern "C"
