// Tensor-core batches: a sequence of Ozaki INT8 or 3xTF32 contractions on one
// stream with one shared workspace (the instances of the configurations this
// serves, m, n <= 1024 and k ~ 1.5e5, each fill all SMs on their own), captured
// into a CUDA graph and replayed. The grouped single-launch form of the batch
// is the FP64 kernel's (gemm_dmma.cu); the residue and TF32 planes of a whole
// batch would not fit in device memory at once, so here the planes of one
// instance are built, consumed and overwritten by the next.
#include <algorithm>
#include <vector>

#include "batch_seq.cuh"
#include "common.cuh"
#include "ozaki.cuh"
#include "splab.h"
#include "tf32x3.cuh"

namespace splab {

struct SeqBatch {
  int path = 0;
  std::vector<GemmProblem> probs;
  size_t ws_bytes = 0;     // shared by all instances
  size_t off_status = 0;   // batch status word after the shared part
  size_t total = 0;
  bool ran_once = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void* graph_ws = nullptr;
  cudaStream_t own = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
};

namespace {

__global__ void or_status_kernel(const int* __restrict__ src, int* __restrict__ dst) {
  if (*src) *dst = 1;
}

size_t instance_ws(int path, const GemmProblem& p) {
  return path == SPLAB_PATH_OZAKI ? ozaki_workspace_bytes(p, 0) : tf32x3_workspace_bytes(p);
}

// The sequence: clear the batch status, then per instance the contraction and
// the or of its status word into the batch status.
cudaError_t enqueue(SeqBatch& b, char* ws, cudaStream_t st) {
  int* bstatus = reinterpret_cast<int*>(ws + b.off_status);
  cudaError_t e = cudaMemsetAsync(bstatus, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  for (const GemmProblem& p : b.probs) {
    if (b.path == SPLAB_PATH_OZAKI) {
      if ((e = ozaki_gemm(p, 0, ws, b.ws_bytes, st)) != cudaSuccess) return e;
      if (p.k > 0) or_status_kernel<<<1, 1, 0, st>>>(ozaki_status_ptr(p, 0, ws), bstatus);
    } else {
      if ((e = tf32x3_gemm(p, ws, b.ws_bytes, st)) != cudaSuccess) return e;
      if (p.k > 0) or_status_kernel<<<1, 1, 0, st>>>(tf32x3_status_ptr(p, ws), bstatus);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

SeqBatch* seq_batch_create(int path, const std::vector<GemmProblem>& probs) {
  if (path != SPLAB_PATH_OZAKI && path != SPLAB_PATH_TF32X3) return nullptr;
  auto* b = new SeqBatch();
  b->path = path;
  b->probs = probs;
  for (const GemmProblem& p : probs) {
    if (path == SPLAB_PATH_OZAKI ? !ozaki_supported(p) : !tf32x3_supported(p)) {
      delete b;
      return nullptr;
    }
    b->ws_bytes = std::max(b->ws_bytes, instance_ws(path, p));
  }
  b->ws_bytes = (b->ws_bytes + 255) & ~size_t(255);
  b->off_status = b->ws_bytes;
  b->total = b->ws_bytes + 256;
  return b;
}

size_t seq_batch_workspace(const SeqBatch* b) { return b->total; }

cudaError_t seq_batch_run(SeqBatch* b, void* ws, cudaStream_t st) {
  cudaError_t e;
  char* w = static_cast<char*>(ws);
  if (!b->ran_once) {
    // direct run: sets kernel attributes and per-device state outside capture
    if ((e = enqueue(*b, w, st)) != cudaSuccess) return e;
    b->ran_once = true;
    return cudaSuccess;
  }
  if (!b->own) {
    if ((e = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming)) != cudaSuccess) return e;
    if ((e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming)) != cudaSuccess)
      return e;
  }
  if (!b->exec || b->graph_ws != ws) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    // no side streams and no phase events inside the captured sequence
    PhaseEvents saved = phase_events();
    phase_events() = PhaseEvents{};
    ozaki_allow_side_streams(false);
    if ((e = cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
      ozaki_allow_side_streams(true);
      phase_events() = saved;
      return e;
    }
    const cudaError_t e1 = enqueue(*b, w, b->own);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->own, &g);
    ozaki_allow_side_streams(true);
    phase_events() = saved;
    if (e1 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return e1;
    }
    if (e != cudaSuccess) return e;
    b->graph = g;
    if ((e = cudaGraphInstantiate(&b->exec, g, 0)) != cudaSuccess) return e;
    b->graph_ws = ws;
  }
  if ((e = cudaEventRecord(b->ev_in, st)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(b->own, b->ev_in, 0)) != cudaSuccess) return e;
  if ((e = cudaGraphLaunch(b->exec, b->own)) != cudaSuccess) return e;
  if ((e = cudaEventRecord(b->ev_out, b->own)) != cudaSuccess) return e;
  return cudaStreamWaitEvent(st, b->ev_out, 0);
}

int seq_batch_status(SeqBatch* b, void* ws, cudaStream_t st) {
  int h = 0;
  cudaMemcpyAsync(&h, static_cast<char*>(ws) + b->off_status, sizeof(int),
                  cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return h;
}

void seq_batch_destroy(SeqBatch* b) {
  if (!b) return;
  if (b->own) cudaStreamSynchronize(b->own);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->ev_in) cudaEventDestroy(b->ev_in);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
}

}  // namespace splab
