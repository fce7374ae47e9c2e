// ctx.h -- internal: the context object behind nrg_ctx* and the host helpers shared by
// the C-ABI layer and the launch planners (workspace arena, descriptor staging, GEMM plans).
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "nrg_b200.h"
#include "kernels.h"

namespace nrg {
// Launch groups timed by nrg_profile (names in phase_name()).
enum Phase : int {
  kPhEigSmall, kPhTridiag, kPhDcLeaf, kPhDcPrep, kPhDcSecular, kPhDcVectors, kPhDcGemm, kPhSort, kPhBtGemm,
  kPhBtTfactor, kPhGemm3, kPhSpecGemm, kPhSpecBin, kPhAssemble, kPhBroaden, kPhBandReduce, kPhBulgeChase,
  kPhBtBand, kPhBandPanel, kPhCount
};
const char* phase_name(int p);
}  // namespace nrg

struct nrg_ctx {
  int device = 0;
  nrg_tuning tune = {nrg::kSmallMaxN, nrg::kMidMaxN, nrg::kClusterMaxN, 3, 3072, 64};  // the autotuner's B200 values
  // profiling: launch counts per phase (always), CUDA-event intervals (when enabled)
  bool prof = false;
  long long launches[nrg::kPhCount] = {};
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct Mark { int phase, b, e; };
  std::vector<Mark> marks;
  size_t ws_limit = 0;
  void* ws = nullptr;  // device workspace arena (grow-only)
  size_t ws_size = 0;
  void* desc = nullptr;  // device copy of launch descriptors
  size_t desc_size = 0;
  int* info_dev = nullptr;
  size_t info_cap = 0;
  // second stream: the one-CTA small-block solver runs beside the large-block pipeline
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  void* desc_side = nullptr;  // descriptor staging of the side stream
  size_t desc_side_size = 0;
  // third stream: the one-CTA tridiagonalisation of mid-size blocks beside the cluster and
  // bulk-copy reductions of larger blocks
  cudaStream_t side2 = nullptr;
  cudaEvent_t fork2_ev = nullptr, join2_ev = nullptr;
  // fourth stream: the two-stage reduction of the largest blocks beside the one-stage ones
  cudaStream_t side3 = nullptr;
  cudaEvent_t fork3_ev = nullptr, join3_ev = nullptr;
  // Cross-stream order of calls: every entry point records order_ev on its stream when it
  // leaves; a call on another stream first waits for it, so the descriptor staging buffers
  // and the workspace arena are never rewritten while an earlier call's kernels read them.
  cudaEvent_t order_ev = nullptr;
  cudaStream_t order_stream = nullptr;
  bool order_set = false;
  // nrg_diag_batch_host: ring of device slots for streamed chunks of blocks, and the two
  // copy streams (host to device, device to host) beside the compute stream
  void* ring = nullptr;
  size_t ring_size = 0;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t ring_ev[3][3] = {};  // per slot: inputs copied, solved, outputs copied
};

namespace nrg {

int fail(int code, const char* fmt, ...);
const char* last_error_text();
int ensure_ws(nrg_ctx* c, size_t bytes);
// Bytes the workspace arena may hold now (context limit, free device memory, a reserve).
size_t ws_available(nrg_ctx* c);
// Copies a host byte image to c->desc (stream-ordered); returns the device base pointer.
int stage_desc(nrg_ctx* c, const std::vector<char>& img, cudaStream_t s);
// Same into the side stream's own staging buffer.
int stage_desc_side(nrg_ctx* c, const std::vector<char>& img);

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename T>
size_t push(std::vector<char>& img, const std::vector<T>& v) {
  const size_t off = align_up(img.size(), 256);
  img.resize(off + sizeof(T) * v.size());
  if (!v.empty()) std::memcpy(img.data() + off, v.data(), sizeof(T) * v.size());
  return off;
}

struct GemmPlan {
  std::vector<GemmOut> outs;
  std::vector<GemmSeg> segs;
  int tiles = 0;
  void add_out(double* C, int64_t ldc, int M, int N, double beta);
  void add_seg(const double* A, int64_t lda, int transA, const double* B, int64_t ldb, int transB, int K,
               double alpha);
};

// Stage the plan's descriptors into `img` (offsets returned) -- used when several plans
// and other descriptors share one staging copy.
struct StagedGemm {
  size_t outs_off = 0, segs_off = 0;
  int nout = 0, tiles = 0;
};
StagedGemm stage_gemm(std::vector<char>& img, const GemmPlan& p);
int launch_staged_gemm(nrg_ctx* c, const StagedGemm& g, cudaStream_t s, int phase);

int run_gemm_plan(nrg_ctx* c, const GemmPlan& p, cudaStream_t s, int phase);

// Orders an entry point's work on stream s after the previous call on the context (on
// whatever stream that ran) and records the point the next call waits for.
struct CallOrder {
  nrg_ctx* c;
  cudaStream_t s;
  CallOrder(nrg_ctx* c_, cudaStream_t s_) : c(c_), s(s_) {
    if (c->order_set && c->order_stream != s) cudaStreamWaitEvent(s, c->order_ev, 0);
  }
  ~CallOrder() {
    if (!c->order_ev && cudaEventCreateWithFlags(&c->order_ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      c->order_ev = nullptr;
      return;
    }
    if (cudaEventRecord(c->order_ev, s) == cudaSuccess) {
      c->order_stream = s;
      c->order_set = true;
    } else {
      cudaGetLastError();
    }
  }
};

// Counts `nlaunch` kernel launches of `phase` and, when profiling, brackets them with
// CUDA events recorded on stream s.
struct PhaseScope {
  nrg_ctx* c;
  cudaStream_t s;
  int mark = -1;
  PhaseScope(nrg_ctx* c, int phase, cudaStream_t s, int nlaunch = 1);
  ~PhaseScope();
};

}  // namespace nrg

#define NRG_CK(call)                                                                                      \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess)                                                                                \
      return ::nrg::fail(NRG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)
