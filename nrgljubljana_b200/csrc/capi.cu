// capi.cu -- the C-ABI of the NRG step core (include/nrg_b200.h): context, device
// workspace, descriptor staging and the host-side planning of every batched launch.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "nrg_b200.h"
#include "ctx.h"
#include "eig_large.h"
#include "kernels.h"
#include "spec.h"

namespace nrg {

namespace {
thread_local std::string g_err;
}

const char* last_error_text() { return g_err.c_str(); }

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

size_t ws_available(nrg_ctx* c) {
  // What the arena may grow to now: the context's limit, and no more than the memory free on
  // the device (plus the arena itself) less a reserve of 2 GiB or 2% of the device, so that the
  // caller's own allocations (a run's growing set of stored eigenvectors) keep room.
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return std::min(c->ws_limit, c->ws_size);
  }
  const size_t reserve = std::max<size_t>((size_t)2 << 30, tot / 50);
  const size_t have = fr + c->ws_size;
  return std::min(c->ws_limit, have > reserve ? have - reserve : c->ws_size);
}

int ensure_ws(nrg_ctx* c, size_t bytes) {
  if (bytes <= c->ws_size) return NRG_OK;
  const size_t lim = ws_available(c);
  if (bytes > lim)
    return fail(NRG_ERR_OOM, "workspace of %zu bytes exceeds the %zu bytes the context can use now", bytes, lim);
  if (c->ws) {
    NRG_CK(cudaDeviceSynchronize());
    NRG_CK(cudaFree(c->ws));
    c->ws = nullptr;
    c->ws_size = 0;
  }
  const size_t sz = std::max(bytes, std::min(lim, align_up(bytes + bytes / 4, 1 << 20)));
  if (cudaMalloc(&c->ws, sz) != cudaSuccess) {
    cudaGetLastError();
    if (cudaMalloc(&c->ws, bytes) != cudaSuccess) {
      cudaGetLastError();
      c->ws = nullptr;
      return fail(NRG_ERR_OOM, "cudaMalloc of %zu bytes of workspace failed", bytes);
    }
    c->ws_size = bytes;
  } else {
    c->ws_size = sz;
  }
  return NRG_OK;
}

// The host image is pageable, so the copy has left it when cudaMemcpyAsync returns.
int stage_desc(nrg_ctx* c, const std::vector<char>& img, cudaStream_t s) {
  if (img.empty()) return NRG_OK;
  if (img.size() > c->desc_size) {
    if (c->desc) {
      NRG_CK(cudaDeviceSynchronize());
      NRG_CK(cudaFree(c->desc));
      c->desc = nullptr;
    }
    const size_t sz = align_up(img.size() * 2, 1 << 16);
    NRG_CK(cudaMalloc(&c->desc, sz));
    c->desc_size = sz;
  }
  NRG_CK(cudaMemcpyAsync(c->desc, img.data(), img.size(), cudaMemcpyHostToDevice, s));
  return NRG_OK;
}

void GemmPlan::add_out(double* C, int64_t ldc, int M, int N, double beta) {
  GemmOut o{};
  o.C = C;
  o.ldc = ldc;
  o.M = M;
  o.N = N;
  o.seg0 = (int)segs.size();
  o.nseg = 0;
  o.tile0 = tiles;
  o.beta = beta;
  tiles += ((M + kGemmBM - 1) / kGemmBM) * ((N + kGemmBN - 1) / kGemmBN);
  outs.push_back(o);
}

void GemmPlan::add_seg(const double* A, int64_t lda, int transA, const double* B, int64_t ldb, int transB, int K,
                       double alpha) {
  GemmSeg g{};
  g.A = A;
  g.B = B;
  g.lda = lda;
  g.ldb = ldb;
  g.K = K;
  g.transA = transA;
  g.transB = transB;
  g.alpha = alpha;
  segs.push_back(g);
  outs.back().nseg++;
}

StagedGemm stage_gemm(std::vector<char>& img, const GemmPlan& p) {
  StagedGemm g;
  g.outs_off = push(img, p.outs);
  g.segs_off = push(img, p.segs);
  g.nout = (int)p.outs.size();
  g.tiles = p.tiles;
  return g;
}

int stage_desc_side(nrg_ctx* c, const std::vector<char>& img) {
  if (img.empty()) return NRG_OK;
  if (img.size() > c->desc_side_size) {
    if (c->desc_side) {
      NRG_CK(cudaStreamSynchronize(c->side));
      NRG_CK(cudaFree(c->desc_side));
      c->desc_side = nullptr;
    }
    const size_t sz = align_up(img.size() * 2, 1 << 16);
    NRG_CK(cudaMalloc(&c->desc_side, sz));
    c->desc_side_size = sz;
  }
  NRG_CK(cudaMemcpyAsync(c->desc_side, img.data(), img.size(), cudaMemcpyHostToDevice, c->side));
  return NRG_OK;
}

const char* phase_name(int p) {
  static const char* names[kPhCount] = {"eig_small", "tridiag", "dc_leaf", "dc_prep", "dc_secular",
                                        "dc_vectors", "dc_gemm", "sort", "bt_gemm", "bt_tfactor",
                                        "gemm3", "spec_gemm", "spec_bin", "assemble", "broaden",
                                        "band_reduce", "bulge_chase", "bt_band", "band_panel"};
  return (p >= 0 && p < kPhCount) ? names[p] : "?";
}

static cudaEvent_t take_event(nrg_ctx* c) {
  if (c->ev_used == c->ev_pool.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    c->ev_pool.push_back(e);
  }
  return c->ev_pool[c->ev_used++];
}

PhaseScope::PhaseScope(nrg_ctx* c_, int phase, cudaStream_t s_, int nlaunch) : c(c_), s(s_) {
  c->launches[phase] += nlaunch;
  if (!c->prof) return;
  cudaEvent_t b = take_event(c), e = take_event(c);
  if (!b || !e) return;
  cudaEventRecord(b, s);
  mark = (int)c->marks.size();
  c->marks.push_back(nrg_ctx::Mark{phase, (int)c->ev_used - 2, (int)c->ev_used - 1});
}

PhaseScope::~PhaseScope() {
  if (mark >= 0) cudaEventRecord(c->ev_pool[c->marks[mark].e], s);
}

int launch_staged_gemm(nrg_ctx* c, const StagedGemm& g, cudaStream_t s, int phase) {
  if (g.nout == 0 || g.tiles == 0) return NRG_OK;
  PhaseScope ps(c, phase, s);
  const char* base = static_cast<const char*>(c->desc);
  NRG_CK(gemm_batch_launch(reinterpret_cast<const GemmOut*>(base + g.outs_off),
                           reinterpret_cast<const GemmSeg*>(base + g.segs_off), g.nout, g.tiles, s));
  return NRG_OK;
}

int run_gemm_plan(nrg_ctx* c, const GemmPlan& p, cudaStream_t s, int phase) {
  if (p.outs.empty() || p.tiles == 0) return NRG_OK;
  std::vector<char> img;
  const StagedGemm g = stage_gemm(img, p);
  int rc = stage_desc(c, img, s);
  if (rc) return rc;
  return launch_staged_gemm(c, g, s, phase);
}

}  // namespace nrg

namespace {
using nrg::fail;
using nrg::ensure_ws;
using nrg::stage_desc;
using nrg::push;
using nrg::GemmPlan;
using nrg::run_gemm_plan;
#define CK NRG_CK

int check_ctx(nrg_ctx* c) {
  if (!c) return fail(NRG_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  return NRG_OK;
}
}  // namespace

extern "C" {

int nrg_version(void) { return NRG_B200_VERSION; }

const char* nrg_last_error(void) { return nrg::last_error_text(); }

int nrg_create(nrg_ctx** out, int device, size_t workspace_limit) {
  if (!out) return fail(NRG_ERR_ARG, "null output pointer");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(NRG_ERR_NODEV, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(NRG_ERR_ARG, "device %d out of range [0,%d)", device, ndev);
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return fail(NRG_ERR_NODEV, "device %d is sm_%d%d; this library is built for sm_100a", device,
                                    prop.major, prop.minor);
  CK(cudaSetDevice(device));
  auto* c = new nrg_ctx();
  c->device = device;
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  c->ws_limit = workspace_limit ? workspace_limit : (size_t)(0.9 * (double)fr);
  *out = c;
  return NRG_OK;
}

int nrg_get_tuning(nrg_ctx* c, nrg_tuning* out) {
  if (!c || !out) return fail(NRG_ERR_ARG, "bad arguments");
  *out = c->tune;
  return NRG_OK;
}

int nrg_set_tuning(nrg_ctx* c, const nrg_tuning* in) {
  if (!c || !in) return fail(NRG_ERR_ARG, "bad arguments");
  const nrg_tuning t = *in;
  if (t.small_max_n < 32 || t.small_max_n > nrg::kSmallMaxNLimit)
    return fail(NRG_ERR_ARG, "small_max_n = %d outside [32, %d]", t.small_max_n, nrg::kSmallMaxNLimit);
  if (t.mid_max_n < t.small_max_n || t.mid_max_n > nrg::kMidMaxNLimit)
    return fail(NRG_ERR_ARG, "mid_max_n = %d outside [small_max_n, %d]", t.mid_max_n, nrg::kMidMaxNLimit);
  if (t.cluster_max_n < t.mid_max_n || t.cluster_max_n > nrg::kClusterMaxNLimit)
    return fail(NRG_ERR_ARG, "cluster_max_n = %d outside [mid_max_n, %d]", t.cluster_max_n,
                nrg::kClusterMaxNLimit);
  if (t.reduction_ctas_per_sm < 1 || t.reduction_ctas_per_sm > 3)
    return fail(NRG_ERR_ARG, "reduction_ctas_per_sm = %d (1, 2 or 3)", t.reduction_ctas_per_sm);
  if (t.band_min_n != 0 && (t.band_min_n < 256 || t.band_min_n > NRG_DIAG_MAX_N))
    return fail(NRG_ERR_ARG, "band_min_n = %d (0, or 256 .. %d)", t.band_min_n, NRG_DIAG_MAX_N);
  if (t.band_max_blocks < 1) return fail(NRG_ERR_ARG, "band_max_blocks = %d (at least 1)", t.band_max_blocks);
  c->tune = t;
  return NRG_OK;
}

int nrg_profile(nrg_ctx* c, int enable) {
  if (!c) return fail(NRG_ERR_ARG, "null context");
  CK(cudaSetDevice(c->device));
  if (enable) {
    CK(cudaDeviceSynchronize());
    c->marks.clear();
    c->ev_used = 0;
    for (auto& l : c->launches) l = 0;
  }
  c->prof = enable != 0;
  return NRG_OK;
}

int nrg_profile_read(nrg_ctx* c, nrg_phase_stat* out, int max) {
  if (!c || (max > 0 && !out)) return fail(NRG_ERR_ARG, "bad arguments");
  CK(cudaSetDevice(c->device));
  double ms[nrg::kPhCount] = {};
  for (const auto& m : c->marks) {
    CK(cudaEventSynchronize(c->ev_pool[m.e]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->ev_pool[m.b], c->ev_pool[m.e]));
    ms[m.phase] += t;
  }
  int k = 0;
  for (int p = 0; p < nrg::kPhCount && k < max; p++) {
    if (c->launches[p] == 0) continue;
    std::snprintf(out[k].name, sizeof out[k].name, "%s", nrg::phase_name(p));
    out[k].ms = ms[p];
    out[k].launches = c->launches[p];
    k++;
  }
  return k;
}

int nrg_destroy(nrg_ctx* c) {
  if (!c) return NRG_OK;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->ws) cudaFree(c->ws);
  if (c->desc) cudaFree(c->desc);
  if (c->info_dev) cudaFree(c->info_dev);
  if (c->desc_side) cudaFree(c->desc_side);
  if (c->fork_ev) cudaEventDestroy(c->fork_ev);
  if (c->join_ev) cudaEventDestroy(c->join_ev);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->fork2_ev) cudaEventDestroy(c->fork2_ev);
  if (c->join2_ev) cudaEventDestroy(c->join2_ev);
  if (c->side2) cudaStreamDestroy(c->side2);
  if (c->fork3_ev) cudaEventDestroy(c->fork3_ev);
  if (c->join3_ev) cudaEventDestroy(c->join3_ev);
  if (c->side3) cudaStreamDestroy(c->side3);
  if (c->ring) cudaFree(c->ring);
  if (c->copy_in) cudaStreamDestroy(c->copy_in);
  if (c->copy_out) cudaStreamDestroy(c->copy_out);
  for (auto& sl : c->ring_ev)
    for (auto e : sl)
      if (e) cudaEventDestroy(e);
  if (c->order_ev) cudaEventDestroy(c->order_ev);
  delete c;
  return NRG_OK;
}

// ---------------------------------------------------------------- diagonalisation
int nrg_diag_batch(nrg_ctx* c, int nblk, const int* n, double* const* H, double* const* evals, double* const* evecs,
                   int* info, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nblk < 0 || (nblk > 0 && (!n || !H || !evals || !evecs || !info))) return fail(NRG_ERR_ARG, "bad arguments");
  if (nblk == 0) return NRG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  for (int b = 0; b < nblk; b++) {
    if (n[b] < 1 || n[b] > NRG_DIAG_MAX_N) return fail(NRG_ERR_ARG, "block %d: order %d out of range", b, n[b]);
    if (!H[b] || !evals[b] || !evecs[b]) return fail(NRG_ERR_ARG, "block %d: null pointer", b);
    if (H[b] == evecs[b]) return fail(NRG_ERR_ARG, "block %d: evecs aliases H", b);
  }
  if ((size_t)nblk > c->info_cap) {
    if (c->info_dev) CK(cudaFree(c->info_dev));
    CK(cudaMalloc(&c->info_dev, sizeof(int) * (size_t)nblk));
    c->info_cap = nblk;
  }
  CK(cudaMemsetAsync(c->info_dev, 0, sizeof(int) * (size_t)nblk, s));

  std::vector<int> small, large;
  for (int b = 0; b < nblk; b++) (n[b] <= c->tune.small_max_n ? small : large).push_back(b);

  // With blocks of both kinds the small-block solver runs on the context's side stream,
  // forked from and joined back into s, so that it overlaps the large-block pipeline.
  const bool fork = !small.empty() && !large.empty();
  if (fork && !c->side) {
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming));
  }
  if (!small.empty()) {
    // Largest first, so that the long CTAs start early.
    std::stable_sort(small.begin(), small.end(), [n](int a, int b) { return n[a] > n[b]; });
    std::vector<nrg::EigBlock> blk(small.size());
    for (size_t t = 0; t < small.size(); t++) {
      const int b = small[t];
      nrg::EigBlock& e = blk[t];
      std::memset(&e, 0, sizeof e);
      e.H = H[b];
      e.evals = evals[b];
      e.evecs = evecs[b];
      e.info = c->info_dev + b;
      e.n = n[b];
    }
    std::vector<char> img;
    const size_t off = push(img, blk);
    cudaStream_t ss = s;
    char* base;
    if (fork) {
      CK(cudaEventRecord(c->fork_ev, s));
      CK(cudaStreamWaitEvent(c->side, c->fork_ev, 0));
      ss = c->side;
      rc = nrg::stage_desc_side(c, img);
      base = static_cast<char*>(c->desc_side);
    } else {
      rc = stage_desc(c, img, s);
      base = static_cast<char*>(c->desc);
    }
    if (rc) return rc;
    {
      nrg::PhaseScope ps(c, nrg::kPhEigSmall, ss);
      CK(nrg::eig_small_launch(reinterpret_cast<const nrg::EigBlock*>(base + off), (int)small.size(),
                               n[small[0]], ss));
    }
    if (fork) CK(cudaEventRecord(c->join_ev, ss));
  }
  if (!large.empty()) {
    rc = nrg::eig_large_run(c, large, n, H, evals, evecs, c->info_dev, s);
    if (fork) {
      const cudaError_t e = cudaStreamWaitEvent(s, c->join_ev, 0);  // join even on failure
      if (!rc && e != cudaSuccess) rc = fail(NRG_ERR_CUDA, "join of the side stream: %s", cudaGetErrorString(e));
    }
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(info, c->info_dev, sizeof(int) * (size_t)nblk, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  int bad = 0;
  for (int b = 0; b < nblk; b++) bad += info[b] != 0;
  if (bad) fail(bad, "%d of %d blocks returned a non-zero status", bad, nblk);
  return bad;
}

int nrg_diag_batch_host(nrg_ctx* c, int nblk, const int* n, const double* const* H, double* const* evals,
                        double* const* evecs, int* info, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nblk < 0 || (nblk > 0 && (!n || !H || !evals || !evecs || !info))) return fail(NRG_ERR_ARG, "bad arguments");
  if (nblk == 0) return NRG_OK;
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  // Device bytes of one block in a ring slot: H and evecs (n^2 each) and evals.
  auto slot_bytes = [&](int b) {
    return 2 * nrg::align_up(sizeof(double) * (size_t)n[b] * n[b], 256) + nrg::align_up(sizeof(double) * n[b], 256);
  };
  size_t total = 0;
  for (int b = 0; b < nblk; b++) {
    if (n[b] < 1 || n[b] > NRG_DIAG_MAX_N) return fail(NRG_ERR_ARG, "block %d: order %d out of range", b, n[b]);
    if (!H[b] || !evals[b] || !evecs[b]) return fail(NRG_ERR_ARG, "block %d: null pointer", b);
    total += slot_bytes(b);
  }
  // Chunks of consecutive blocks stream through a ring of up to three device slots: the
  // host-to-device copy of chunk k+1 and the device-to-host copy of chunk k-1 run on two
  // copy streams beside the solve of chunk k. A slot holds about half of the batch, at most
  // 32 GiB, and at most a fifth of the memory this context can use (the solve's own workspace
  // comes on top of the slots). Few large chunks keep each solve's batch wide enough to fill
  // the SMs: every chunk ends in a tail where its largest blocks hold few of them.
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  const size_t usable = std::min(c->ws_limit, fr + c->ring_size + c->ws_size);
  size_t target = std::min<size_t>(std::max<size_t>(total / 2 + 1, (size_t)64 << 20), (size_t)32 << 30);
  target = std::max<size_t>(std::min(target, usable / 5), (size_t)16 << 20);
  std::vector<int> first(1, 0);
  size_t maxchunk = 0, cur = 0;
  for (int b = 0; b < nblk; b++) {
    const size_t sb = slot_bytes(b);
    if (b > first.back() && cur + sb > target) {
      maxchunk = std::max(maxchunk, cur);
      first.push_back(b);
      cur = 0;
    }
    cur += sb;
  }
  maxchunk = std::max(maxchunk, cur);
  first.push_back(nblk);
  const int nchunk = (int)first.size() - 1;
  const int nslot = std::min(3, nchunk);
  const size_t slot = nrg::align_up(maxchunk, 1 << 20);
  if (c->ring_size < slot * nslot) {
    if (c->ring) {
      CK(cudaDeviceSynchronize());
      CK(cudaFree(c->ring));
      c->ring = nullptr;
      c->ring_size = 0;
    }
    if (cudaMalloc(&c->ring, slot * nslot) != cudaSuccess) {
      cudaGetLastError();
      c->ring = nullptr;
      return fail(NRG_ERR_OOM, "device ring of %d slots of %zu bytes for the host blocks", nslot, slot);
    }
    c->ring_size = slot * nslot;
  }
  if (!c->copy_in) {
    CK(cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking));
    for (auto& sl : c->ring_ev)
      for (auto& e : sl) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  // Device pointers of every block inside its chunk's slot.
  std::vector<double*> pH(nblk), pV(nblk), pE(nblk);
  for (int k = 0; k < nchunk; k++) {
    char* base = static_cast<char*>(c->ring) + (size_t)(k % nslot) * slot;
    size_t off = 0;
    for (int b = first[k]; b < first[k + 1]; b++) {
      const size_t m = nrg::align_up(sizeof(double) * (size_t)n[b] * n[b], 256);
      pH[b] = reinterpret_cast<double*>(base + off);
      pV[b] = reinterpret_cast<double*>(base + off + m);
      pE[b] = reinterpret_cast<double*>(base + off + 2 * m);
      off += slot_bytes(b);
    }
  }
  auto settle = [&]() {  // no copy may still target the ring or the caller's memory
    const cudaError_t e1 = cudaStreamSynchronize(c->copy_in);
    const cudaError_t e2 = cudaStreamSynchronize(c->copy_out);
    const cudaError_t e3 = cudaStreamSynchronize(s);
    return e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3;
  };
  auto copy_in = [&](int k) -> int {
    const int sl = k % nslot;
    if (k >= nslot) CK(cudaStreamWaitEvent(c->copy_in, c->ring_ev[sl][2], 0));  // chunk k - nslot copied out
    for (int b = first[k]; b < first[k + 1]; b++)
      CK(cudaMemcpyAsync(pH[b], H[b], sizeof(double) * (size_t)n[b] * n[b], cudaMemcpyHostToDevice, c->copy_in));
    CK(cudaEventRecord(c->ring_ev[sl][0], c->copy_in));
    return NRG_OK;
  };
  int bad = 0;
  for (int k = 0; k < nchunk && rc == NRG_OK; k++) {
    if (k == 0) rc = copy_in(0);
    if (rc == NRG_OK && k + 1 < nchunk) rc = copy_in(k + 1);
    if (rc) break;
    const int sl = k % nslot, b0 = first[k], nb = first[k + 1] - b0;
    if (cudaStreamWaitEvent(s, c->ring_ev[sl][0], 0) != cudaSuccess) {
      rc = fail(NRG_ERR_CUDA, "stream wait for the copy of chunk %d", k);
      break;
    }
    const int r = nrg_diag_batch(c, nb, n + b0, pH.data() + b0, pE.data() + b0, pV.data() + b0, info + b0, stream);
    if (r < 0) {
      rc = r;
      break;
    }
    bad += r;
    if (cudaEventRecord(c->ring_ev[sl][1], s) != cudaSuccess ||
        cudaStreamWaitEvent(c->copy_out, c->ring_ev[sl][1], 0) != cudaSuccess) {
      rc = fail(NRG_ERR_CUDA, "ordering of the copy-out of chunk %d", k);
      break;
    }
    for (int b = b0; b < b0 + nb && rc == NRG_OK; b++) {
      if (cudaMemcpyAsync(evals[b], pE[b], sizeof(double) * n[b], cudaMemcpyDeviceToHost, c->copy_out) != cudaSuccess ||
          cudaMemcpyAsync(evecs[b], pV[b], sizeof(double) * (size_t)n[b] * n[b], cudaMemcpyDeviceToHost,
                          c->copy_out) != cudaSuccess)
        rc = fail(NRG_ERR_CUDA, "copy-out of block %d", b);
    }
    if (rc == NRG_OK && cudaEventRecord(c->ring_ev[sl][2], c->copy_out) != cudaSuccess)
      rc = fail(NRG_ERR_CUDA, "event after the copy-out of chunk %d", k);
  }
  const cudaError_t se = settle();
  if (rc == NRG_OK && se != cudaSuccess)
    rc = fail(NRG_ERR_CUDA, "copies of the host blocks: %s", cudaGetErrorString(se));
  if (rc) return rc;
  if (bad) fail(bad, "%d of %d blocks returned a non-zero status", bad, nblk);
  return bad;
}

int nrg_trim(nrg_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CK(cudaDeviceSynchronize());
  if (c->ws) CK(cudaFree(c->ws));
  c->ws = nullptr;
  c->ws_size = 0;
  if (c->ring) CK(cudaFree(c->ring));
  c->ring = nullptr;
  c->ring_size = 0;
  if (c->desc) CK(cudaFree(c->desc));
  c->desc = nullptr;
  c->desc_size = 0;
  if (c->desc_side) CK(cudaFree(c->desc_side));
  c->desc_side = nullptr;
  c->desc_side_size = 0;
  return NRG_OK;
}

// ---------------------------------------------------------------- GEMM leaves
int nrg_hamiltonian_batch(nrg_ctx* c, int nblk, const int* n, double* const* H, int npiece,
                          const nrg_hpiece* pieces, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nblk < 0 || npiece < 0 || (nblk > 0 && (!n || !H)) || (npiece > 0 && !pieces))
    return fail(NRG_ERR_ARG, "bad arguments");
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  for (int b = 0; b < nblk; b++) {
    if (n[b] < 0 || n[b] > (1 << 20)) return fail(NRG_ERR_ARG, "block %d: bad order %d", b, n[b]);
    if (n[b] > 0 && !H[b]) return fail(NRG_ERR_ARG, "block %d: null matrix", b);
  }
  for (int p = 0; p < npiece; p++) {
    const nrg_hpiece& q = pieces[p];
    if (q.blk < 0 || q.blk >= nblk) return fail(NRG_ERR_ARG, "piece %d: block %d out of range", p, q.blk);
    const int nb = n[q.blk];
    if (q.kind != NRG_HP_DIAG && q.kind != NRG_HP_BLOCK) return fail(NRG_ERR_ARG, "piece %d: bad kind", p);
    const int cols = q.kind == NRG_HP_DIAG ? q.rows : q.cols;
    if (q.rows < 0 || cols < 0 || q.r0 < 0 || q.c0 < 0 || q.r0 + q.rows > nb || q.c0 + cols > nb)
      return fail(NRG_ERR_ARG, "piece %d: region outside the %d x %d block", p, nb, nb);
    if (!(q.factor - q.factor == 0.0) || !(q.shift - q.shift == 0.0))
      return fail(NRG_ERR_ARG, "piece %d: factor not finite", p);  // c++/matrix.hpp:40-41
    if (q.kind == NRG_HP_BLOCK && q.rows > 0 && q.cols > 0) {
      if (!q.src) return fail(NRG_ERR_ARG, "piece %d: null source matrix", p);
      if (q.ld < (q.trans ? q.rows : q.cols)) return fail(NRG_ERR_ARG, "piece %d: leading dimension too small", p);
    }
  }
  // Pieces grouped by block, order inside a block kept.
  std::vector<int> count(nblk + 1, 0);
  for (int p = 0; p < npiece; p++) count[pieces[p].blk + 1]++;
  for (int b = 0; b < nblk; b++) count[b + 1] += count[b];
  std::vector<nrg_hpiece> sorted(npiece);
  {
    std::vector<int> fill(count.begin(), count.end() - 1);
    for (int p = 0; p < npiece; p++) sorted[fill[pieces[p].blk]++] = pieces[p];
  }
  std::vector<nrg::HBlock> blocks;
  int tiles = 0;
  for (int b = 0; b < nblk; b++) {
    if (n[b] == 0) continue;
    nrg::HBlock hb;
    hb.H = H[b];
    hb.n = n[b];
    hb.tile0 = tiles;
    hb.p0 = count[b];
    hb.p1 = count[b + 1];
    blocks.push_back(hb);
    tiles += nrg::hamiltonian_tiles(n[b]);
  }
  if (blocks.empty()) return NRG_OK;
  std::vector<char> img;
  const size_t ob = push(img, blocks);
  const size_t op = push(img, sorted);
  rc = stage_desc(c, img, s);
  if (rc) return rc;
  auto* base = static_cast<char*>(c->desc);
  nrg::PhaseScope ps(c, nrg::kPhAssemble, s);
  CK(nrg::hamiltonian_launch(reinterpret_cast<const nrg::HBlock*>(base + ob), (int)blocks.size(), tiles,
                             reinterpret_cast<const nrg_hpiece*>(base + op), s));
  return NRG_OK;
}

int nrg_gemm3_batch(nrg_ctx* c, int nterm, const nrg_gemm3* terms, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nterm < 0 || (nterm > 0 && !terms)) return fail(NRG_ERR_ARG, "bad arguments");
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  // Group by output pointer, keeping the given order inside a group.
  std::vector<int> live;
  for (int t = 0; t < nterm; t++) {
    const nrg_gemm3& g = terms[t];
    if (g.rows < 0 || g.cols < 0 || g.ka < 0 || g.kb < 0) return fail(NRG_ERR_ARG, "term %d: negative size", t);
    if (g.rows == 0 || g.cols == 0 || g.ka == 0 || g.kb == 0) continue;
    if (!g.M || !g.A || !g.B) return fail(NRG_ERR_ARG, "term %d: null pointer", t);
    if ((!g.O || g.ldo == 0) && g.ka != g.kb)
      return fail(NRG_ERR_ARG, "term %d: an identity or diagonal O needs ka == kb", t);
    if (g.O && g.ldo != 0 && g.ldo < g.kb) return fail(NRG_ERR_ARG, "term %d: ldo < kb", t);
    if (!(g.factor == g.factor) || g.factor - g.factor != 0.0)
      return fail(NRG_ERR_ARG, "term %d: non-finite factor", t);  // my_assert(my_isfinite(factor))
    live.push_back(t);
  }
  if (live.empty()) return NRG_OK;
  std::map<double*, std::vector<int>> groups;
  std::vector<double*> order;
  for (int t : live) {
    auto& v = groups[terms[t].M];
    if (v.empty()) order.push_back(terms[t].M);
    else {
      const nrg_gemm3& f = terms[v[0]];
      if (f.rows != terms[t].rows || f.cols != terms[t].cols || f.ldm != terms[t].ldm)
        return fail(NRG_ERR_ARG, "term %d: shape of M differs from term %d with the same M", t, v[0]);
    }
    v.push_back(t);
  }
  // Phase 1: T_t = O_t op(B_t) (ka x cols) for every term with an O: a GEMM for a dense O, a
  // row scaling for a diagonal one (ldo == 0). Phase 2: M += sum_t factor_t op(A_t) T_t.
  // The T_t of all terms share the workspace arena; when they do not fit in what the arena may
  // hold now, the output groups (and, for a group too large by itself, its terms) go in
  // consecutive passes on the stream, each adding its terms into M.
  auto tsize = [&](int t) -> size_t { return terms[t].O ? (size_t)terms[t].ka * terms[t].cols : 0; };
  std::vector<std::vector<int>> glist;
  size_t need = 0;
  for (double* M : order) {
    glist.push_back(groups[M]);
    for (int t : glist.back()) need += tsize(t);
  }
  std::vector<std::vector<std::vector<int>>> passes;
  const size_t cap = std::max(c->ws_size, nrg::ws_available(c)) / sizeof(double);
  if (need <= cap) {
    passes.push_back(std::move(glist));
  } else {
    std::vector<std::vector<int>> cur;
    size_t used = 0;
    auto close = [&]() {
      if (!cur.empty()) passes.push_back(std::move(cur));
      cur.clear();
      used = 0;
    };
    for (auto& v : glist) {
      size_t gv = 0;
      for (int t : v) gv += tsize(t);
      if (gv <= cap) {
        if (used + gv > cap) close();
        cur.push_back(v);
        used += gv;
        continue;
      }
      std::vector<int> part;
      for (int t : v) {
        const size_t x = tsize(t);
        if (x > cap)
          return fail(NRG_ERR_OOM, "term %d: workspace of %zu bytes exceeds the %zu bytes the context can use now",
                      t, sizeof(double) * x, sizeof(double) * cap);
        if (used + x > cap) {
          if (!part.empty()) cur.push_back(part);
          part.clear();
          close();
        }
        part.push_back(t);
        used += x;
      }
      if (!part.empty()) cur.push_back(part);
    }
    close();
  }
  auto dense_O = [&](int t) { return terms[t].O && terms[t].ldo != 0; };
  std::vector<size_t> toff(nterm, 0);
  for (const auto& pass : passes) {
    size_t pneed = 0;
    for (const auto& v : pass)
      for (int t : v)
        if (terms[t].O) {
          toff[t] = pneed;
          pneed += tsize(t);
        }
    rc = ensure_ws(c, sizeof(double) * std::max<size_t>(pneed, 1));
    if (rc) return rc;
    double* T = static_cast<double*>(c->ws);
    GemmPlan p1, p2;
    std::vector<nrg::RowScale> rsc;
    int64_t rtotal = 0;
    for (const auto& v : pass)
      for (int t : v) {
        const nrg_gemm3& g = terms[t];
        if (!g.O) continue;
        if (dense_O(t)) {
          p1.add_out(T + toff[t], g.cols, g.ka, g.cols, 0.0);
          p1.add_seg(g.O, g.ldo, 0, g.B, g.ldb, g.transB, g.kb, 1.0);
          continue;
        }
        nrg::RowScale r{};
        r.T = T + toff[t];
        r.d = g.O;
        r.B = g.B;
        r.ldb = g.ldb;
        r.off = rtotal;
        r.rows = g.ka;
        r.cols = g.cols;
        r.transB = g.transB;
        rsc.push_back(r);
        rtotal += (int64_t)g.ka * g.cols;
      }
    for (const auto& v : pass) {
      const nrg_gemm3& f = terms[v[0]];
      p2.add_out(f.M, f.ldm, f.rows, f.cols, 1.0);
      for (int t : v) {
        const nrg_gemm3& g = terms[t];
        if (g.O) p2.add_seg(g.A, g.lda, g.transA, T + toff[t], g.cols, 0, g.ka, g.factor);
        else p2.add_seg(g.A, g.lda, g.transA, g.B, g.ldb, g.transB, g.ka, g.factor);
      }
    }
    if (!rsc.empty()) {
      std::vector<char> img;
      const size_t ro = push(img, rsc);
      rc = stage_desc(c, img, s);
      if (rc) return rc;
      nrg::PhaseScope ps(c, nrg::kPhGemm3, s);
      CK(nrg::row_scale_launch(reinterpret_cast<const nrg::RowScale*>(static_cast<char*>(c->desc) + ro),
                               (int)rsc.size(), rtotal, s));
    }
    rc = run_gemm_plan(c, p1, s, nrg::kPhGemm3);
    if (rc) return rc;
    rc = run_gemm_plan(c, p2, s, nrg::kPhGemm3);
    if (rc) return rc;
  }
  return NRG_OK;
}

int nrg_gemm3_batch_host(nrg_ctx* c, int nterm, const nrg_gemm3* terms, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nterm < 0 || (nterm > 0 && !terms)) return fail(NRG_ERR_ARG, "bad arguments");
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  // Copy every referenced host span once (by pointer), compute, copy M spans back.
  struct Span { size_t bytes; double* dev; };
  std::map<const double*, Span> spans;
  auto span_of = [](const double* p, int r, int cc, int64_t ld) -> size_t {
    return (r == 0 || cc == 0) ? 0 : sizeof(double) * ((size_t)(r - 1) * ld + cc);
  };
  auto note = [&](const double* p, size_t bytes) {
    if (!p || !bytes) return;
    auto it = spans.find(p);
    if (it == spans.end()) spans[p] = Span{bytes, nullptr};
    else it->second.bytes = std::max(it->second.bytes, bytes);
  };
  for (int t = 0; t < nterm; t++) {
    const nrg_gemm3& g = terms[t];
    if (g.rows <= 0 || g.cols <= 0 || g.ka <= 0 || g.kb <= 0) continue;
    note(g.M, span_of(g.M, g.rows, g.cols, g.ldm));
    note(g.A, g.transA ? span_of(g.A, g.ka, g.rows, g.lda) : span_of(g.A, g.rows, g.ka, g.lda));
    if (g.O) note(g.O, g.ldo == 0 ? sizeof(double) * g.ka : span_of(g.O, g.ka, g.kb, g.ldo));
    note(g.B, g.transB ? span_of(g.B, g.cols, g.kb, g.ldb) : span_of(g.B, g.kb, g.cols, g.ldb));
  }
  std::vector<double*> allocs;
  auto cleanup = [&]() { for (double* p : allocs) cudaFree(p); };
  for (auto& kv : spans) {
    double* d = nullptr;
    if (cudaMalloc(&d, kv.second.bytes) != cudaSuccess) {
      cudaGetLastError();
      cleanup();
      return fail(NRG_ERR_OOM, "device copy of %zu bytes", kv.second.bytes);
    }
    allocs.push_back(d);
    kv.second.dev = d;
    cudaMemcpyAsync(d, kv.first, kv.second.bytes, cudaMemcpyHostToDevice, s);
  }
  std::vector<nrg_gemm3> dt(terms, terms + nterm);
  auto dev = [&](const double* p) -> double* { return p ? spans.at(p).dev : nullptr; };
  for (auto& g : dt) {
    if (g.rows <= 0 || g.cols <= 0 || g.ka <= 0 || g.kb <= 0) continue;
    g.M = dev(g.M);
    g.A = dev(g.A);
    g.O = dev(g.O);
    g.B = dev(g.B);
  }
  rc = nrg_gemm3_batch(c, nterm, dt.data(), stream);
  if (rc == NRG_OK) {
    for (int t = 0; t < nterm; t++) {
      const nrg_gemm3& g = terms[t];
      if (g.rows <= 0 || g.cols <= 0 || g.ka <= 0 || g.kb <= 0) continue;
      const Span& sp = spans.at(g.M);
      cudaMemcpyAsync(g.M, sp.dev, sp.bytes, cudaMemcpyDeviceToHost, s);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = fail(NRG_ERR_CUDA, "copy-out failed");
  }
  cleanup();
  return rc;
}

// ---------------------------------------------------------------- spectral accumulation
int nrg_broaden(nrg_ctx* c, int nspike, const double* e, const double* w, int nmesh, const double* E, double alpha,
                double omega0, double* out, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nspike < 0 || nmesh < 0 || (nspike > 0 && (!e || !w)) || (nmesh > 0 && (!E || !out)))
    return fail(NRG_ERR_ARG, "bad arguments");
  if (!(alpha > 0.0) || !(omega0 > 0.0)) return fail(NRG_ERR_ARG, "alpha and omega0 must be positive");
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  nrg::PhaseScope ps(c, nrg::kPhBroaden, s);
  CK(nrg::broaden_launch(nspike, e, w, nmesh, E, alpha, omega0, out, s));
  return NRG_OK;
}

int nrg_bins_grid(const nrg_bins* b, double* energies) {
  if (!b || b->bins <= 0) return fail(NRG_ERR_ARG, "bad bins");
  const int nr = (int)((b->log10emax - b->log10emin) * b->bins + 1.0);
  if (energies)
    for (int i = 0; i < nr; i++) energies[i] = std::pow(10.0, b->log10emin + (double)i / b->bins);
  return nr;
}

int nrg_spec_accumulate(nrg_ctx* c, int npair, const nrg_spec_pair* pairs, const nrg_spec_params* prm,
                        const nrg_bins* bins, double* pos, double* neg, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (npair < 0 || (npair > 0 && (!pairs || !prm || !bins || !pos || !neg))) return fail(NRG_ERR_ARG, "bad arguments");
  if (npair == 0) return NRG_OK;
  if (bins->nbins < 2 || bins->bins <= 0) return fail(NRG_ERR_ARG, "bad bins");
  if (prm->algo < NRG_SPEC_DMNRG || prm->algo > NRG_SPEC_FDMLS) return fail(NRG_ERR_ARG, "bad algo %d", prm->algo);
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);

  // GEMM-derived matrices in workspace.
  std::vector<size_t> xo(npair, 0), yo(npair, 0);
  size_t need = 0;
  for (int p = 0; p < npair; p++) {
    const nrg_spec_pair& q = pairs[p];
    if (q.ni < 0 || q.nj < 0 || q.ki < 0 || q.kj < 0 || q.ki > q.ni || q.kj > q.nj)
      return fail(NRG_ERR_ARG, "pair %d: bad ranges", p);
    if (prm->algo == NRG_SPEC_DMNRG) {
      xo[p] = need; need += (size_t)q.kj * q.ki;
      yo[p] = need; need += (size_t)q.kj * q.ki;
    } else if (prm->algo == NRG_SPEC_FDMGT) {
      if (q.ki > q.rdi) return fail(NRG_ERR_ARG, "pair %d: rdi < ki", p);
      xo[p] = need; need += (size_t)q.nj * q.rdi;
    } else {
      if (q.kj > q.rdj) return fail(NRG_ERR_ARG, "pair %d: rdj < kj", p);
      xo[p] = need; need += (size_t)q.rdj * q.ni;
    }
  }
  rc = ensure_ws(c, sizeof(double) * std::max<size_t>(need, 1));
  if (rc) return rc;
  double* W = static_cast<double*>(c->ws);
  GemmPlan gp;
  std::vector<nrg::SpecRegion> regs;
  auto region = [&](const nrg_spec_pair& q, int kind, int i0, int i1, int j0, int j1, const double* X, int64_t ldx,
                    const double* Y, int64_t ldy, double coef) {
    if (i1 <= i0 || j1 <= j0) return;
    nrg::SpecRegion r{};
    r.Ei = q.Ei; r.Ej = q.Ej; r.op1 = q.op1; r.op2 = q.op2; r.X = X; r.Y = Y;
    r.ld1 = q.ld1; r.ld2 = q.ld2; r.ldx = ldx; r.ldy = ldy;
    r.i0 = i0; r.i1 = i1; r.j0 = j0; r.j1 = j1;
    r.kind = kind; r.sign = prm->sign; r.coef = coef; r.factor = q.factor; r.T = prm->T;
    r.Emin = prm->Emin; r.Emax = prm->Emax;
    regs.push_back(r);
  };
  for (int p = 0; p < npair; p++) {
    const nrg_spec_pair& q = pairs[p];
    if (prm->algo == NRG_SPEC_DMNRG) {
      if (q.ki == 0 || q.kj == 0) continue;
      double* X = W + xo[p];
      double* Y = W + yo[p];
      // X(rj, rm) = sum_ri op2(rj, ri) rho_i(rm, ri)   (algo_DMNRG.hpp:38)
      gp.add_out(X, q.ki, q.kj, q.ki, 0.0);
      gp.add_seg(q.op2, q.ld2, 0, q.rho_i, q.ldri, 1, q.ki, 1.0);
      // Y(rj, rm) = sum_ri rho_j(rj, ri) op1(ri, rm)   (algo_DMNRG.hpp:41)
      gp.add_out(Y, q.ki, q.kj, q.ki, 0.0);
      gp.add_seg(q.rho_j, q.ldrj, 0, q.op1, q.ld1, 0, q.kj, 1.0);
      region(q, nrg::kSpecDMNRG, 0, q.ki, 0, q.kj, X, q.ki, Y, q.ki, 0.0);
    } else if (prm->algo == NRG_SPEC_FDMGT) {
      // op2_rho = prod_fit(op2, rhoFDM(Ii)) (algo_FDM.hpp:89, numerics.hpp:283-306)
      double* X = W + xo[p];
      if (q.rdi > 0 && q.nj > 0) {
        gp.add_out(X, q.rdi, q.nj, q.rdi, 0.0);
        gp.add_seg(q.op2, q.ld2, 0, q.rho_i, q.ldri, 0, std::min(q.rdi, q.ni), 1.0);
      }
      region(q, nrg::kSpecExpI, q.ki, q.ni, 0, q.nj, nullptr, 0, nullptr, 0, prm->wnf);   // D x (D + K)
      region(q, nrg::kSpecGemmX, 0, q.ki, q.kj, q.nj, X, q.rdi, nullptr, 0, 1.0);         // K x D
    } else {
      // rho_op2 = prod_fit(rhoFDM(Ij), op2) (algo_FDM.hpp:35)
      double* X = W + xo[p];
      if (q.rdj > 0 && q.ni > 0) {
        gp.add_out(X, q.ni, q.rdj, q.ni, 0.0);
        gp.add_seg(q.rho_j, q.ldrj, 0, q.op2, q.ld2, 0, std::min(q.rdj, q.nj), 1.0);
      }
      const double ms = (double)(-prm->sign);
      region(q, nrg::kSpecExpJ, 0, q.ni, q.kj, q.nj, nullptr, 0, nullptr, 0, ms * prm->wnf);  // (D + K) x D
      region(q, nrg::kSpecGemmX, q.ki, q.ni, 0, q.kj, X, q.ni, nullptr, 0, ms);                // D x K
    }
  }
  rc = run_gemm_plan(c, gp, s, nrg::kPhSpecGemm);
  if (rc) return rc;
  if (regs.empty()) return NRG_OK;
  std::vector<nrg::SpecTask> tasks;
  const int64_t chunk = 8192;
  for (size_t r = 0; r < regs.size(); r++) {
    const int64_t nt = (int64_t)(regs[r].i1 - regs[r].i0) * (regs[r].j1 - regs[r].j0);
    for (int64_t t0 = 0; t0 < nt; t0 += chunk) {
      nrg::SpecTask k{};
      k.t0 = t0;
      k.t1 = std::min(nt, t0 + chunk);
      k.region = (int)r;
      tasks.push_back(k);
    }
  }
  std::vector<char> img;
  const size_t ro = push(img, regs), to = push(img, tasks);
  rc = stage_desc(c, img, s);
  if (rc) return rc;
  nrg::BinParams bp{};
  bp.log10emin = bins->log10emin;
  bp.discard_immediately = bins->discard_immediately;
  bp.bins = bins->bins;
  bp.nbins = bins->nbins;
  const char* base = static_cast<const char*>(c->desc);
  nrg::PhaseScope ps(c, nrg::kPhSpecBin, s);
  CK(nrg::spec_bin_launch(reinterpret_cast<const nrg::SpecTask*>(base + to), (int)tasks.size(),
                          reinterpret_cast<const nrg::SpecRegion*>(base + ro), bp, pos, neg, s));
  return NRG_OK;
}

int nrg_spec_accumulate_mats(nrg_ctx* c, int npair, const nrg_spec_pair* pairs, const nrg_spec_params* prm,
                             int mats, double* re, double* im, void* stream) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (npair < 0 || (npair > 0 && (!pairs || !prm || !re || !im))) return fail(NRG_ERR_ARG, "bad arguments");
  if (npair == 0) return NRG_OK;
  if (mats < 1 || 2 * sizeof(double) * (size_t)mats > nrg::kSpecSmemMax) return fail(NRG_ERR_ARG, "mats = %d", mats);
  if (!(prm->T > 0.0) || (prm->sign != 1 && prm->sign != -1)) return fail(NRG_ERR_ARG, "bad T or sign");
  const int algo = prm->algo;
  if (algo != NRG_SPEC_DMNRG && algo != NRG_SPEC_FDMMATS && algo != NRG_SPEC_FTMATS)
    return fail(NRG_ERR_ARG, "bad algo %d for the Matsubara sums", algo);
  auto s = static_cast<cudaStream_t>(stream);
  nrg::CallOrder call_order(c, s);
  // FDMmats: op2_rho = prod_fit(op2, rhoFDM(Ii)) (nj x rdi) and rho_op2 = prod_fit(rhoFDM(Ij), op2)
  // (rdj x ni); DMNRGmats: X and Y of the DM-NRG weights (ki x kj... as NRG_SPEC_DMNRG)
  std::vector<size_t> xo(npair, 0), yo(npair, 0);
  size_t need = 0;
  for (int p = 0; p < npair; p++) {
    const nrg_spec_pair& q = pairs[p];
    if (q.ni < 0 || q.nj < 0 || q.ki < 0 || q.kj < 0 || q.ki > q.ni || q.kj > q.nj)
      return fail(NRG_ERR_ARG, "pair %d: bad ranges", p);
    if (algo == NRG_SPEC_DMNRG) {
      xo[p] = need; need += (size_t)q.kj * q.ki;
      yo[p] = need; need += (size_t)q.kj * q.ki;
      continue;
    }
    if (algo == NRG_SPEC_FTMATS) continue;
    if (q.ki > q.rdi || q.kj > q.rdj) return fail(NRG_ERR_ARG, "pair %d: rdi < ki or rdj < kj", p);
    xo[p] = need; need += (size_t)q.nj * q.rdi;
    yo[p] = need; need += (size_t)q.rdj * q.ni;
  }
  rc = ensure_ws(c, sizeof(double) * std::max<size_t>(need, 1));
  if (rc) return rc;
  double* W = static_cast<double*>(c->ws);
  GemmPlan gp;
  std::vector<nrg::SpecRegion> regs;
  auto region = [&](const nrg_spec_pair& q, int kind, int i0, int i1, int j0, int j1, const double* X, int64_t ldx,
                    double coef, int special) {
    if (i1 <= i0 || j1 <= j0) return;
    nrg::SpecRegion r{};
    r.Ei = q.Ei; r.Ej = q.Ej; r.op1 = q.op1; r.op2 = q.op2; r.X = X; r.Y = nullptr;
    r.ld1 = q.ld1; r.ld2 = q.ld2; r.ldx = ldx; r.ldy = 0;
    r.i0 = i0; r.i1 = i1; r.j0 = j0; r.j1 = j1;
    r.kind = kind; r.sign = prm->sign; r.mspecial = special; r.coef = coef; r.factor = q.factor; r.T = prm->T;
    regs.push_back(r);
  };
  const double ms = (double)(-prm->sign);
  for (int p = 0; p < npair; p++) {
    const nrg_spec_pair& q = pairs[p];
    double* X = W + xo[p];
    double* Y = W + yo[p];
    if (algo == NRG_SPEC_DMNRG) {  // Algo_DMNRGmats: the DM-NRG weights over kept x kept, no window
      if (q.ki == 0 || q.kj == 0) continue;
      gp.add_out(X, q.ki, q.kj, q.ki, 0.0);
      gp.add_seg(q.op2, q.ld2, 0, q.rho_i, q.ldri, 1, q.ki, 1.0);
      gp.add_out(Y, q.ki, q.kj, q.ki, 0.0);
      gp.add_seg(q.rho_j, q.ldrj, 0, q.op1, q.ld1, 0, q.kj, 1.0);
      nrg::SpecRegion r{};
      r.Ei = q.Ei; r.Ej = q.Ej; r.op1 = q.op1; r.op2 = q.op2; r.X = X; r.Y = Y;
      r.ld1 = q.ld1; r.ld2 = q.ld2; r.ldx = q.ki; r.ldy = q.ki;
      r.i0 = 0; r.i1 = q.ki; r.j0 = 0; r.j1 = q.kj;
      r.kind = nrg::kSpecDMNRG; r.sign = prm->sign; r.mspecial = nrg::kMatsDmnrgA; r.factor = q.factor;
      r.T = prm->T; r.Emin = -1.0; r.Emax = 1e300;
      regs.push_back(r);
      continue;
    }
    if (algo == NRG_SPEC_FTMATS) {  // Algo_FTmats: the two exponentials over the pair's states
      region(q, nrg::kSpecExpI, 0, q.ni, 0, q.nj, nullptr, 0, prm->wnf, nrg::kMatsZero);
      region(q, nrg::kSpecExpJ, 0, q.ni, 0, q.nj, nullptr, 0, ms * prm->wnf, nrg::kMatsPlusOverT);
      continue;
    }
    if (q.rdi > 0 && q.nj > 0) {
      gp.add_out(X, q.rdi, q.nj, q.rdi, 0.0);
      gp.add_seg(q.op2, q.ld2, 0, q.rho_i, q.ldri, 0, std::min(q.rdi, q.ni), 1.0);
    }
    if (q.rdj > 0 && q.ni > 0) {
      gp.add_out(Y, q.ni, q.rdj, q.ni, 0.0);
      gp.add_seg(q.rho_j, q.ldrj, 0, q.op2, q.ld2, 0, std::min(q.rdj, q.nj), 1.0);
    }
    // term1 (D x D): weightA (exp(-Ei/T)) + weightB (-sign exp(-Ej/T)); term2 (i in D, j in K):
    // weightA + (-sign) op1 rho_op2; term3 (i in K, j in D): op1 op2_rho + weightB
    region(q, nrg::kSpecExpI, q.ki, q.ni, q.kj, q.nj, nullptr, 0, prm->wnf, nrg::kMatsMinusOverT);
    region(q, nrg::kSpecExpJ, q.ki, q.ni, q.kj, q.nj, nullptr, 0, ms * prm->wnf, nrg::kMatsZero);
    region(q, nrg::kSpecExpI, q.ki, q.ni, 0, q.kj, nullptr, 0, prm->wnf, nrg::kMatsPlain);
    region(q, nrg::kSpecGemmX, q.ki, q.ni, 0, q.kj, Y, q.ni, ms, nrg::kMatsPlain);
    region(q, nrg::kSpecGemmX, 0, q.ki, q.kj, q.nj, X, q.rdi, 1.0, nrg::kMatsPlain);
    region(q, nrg::kSpecExpJ, 0, q.ki, q.kj, q.nj, nullptr, 0, ms * prm->wnf, nrg::kMatsPlain);
  }
  rc = run_gemm_plan(c, gp, s, nrg::kPhSpecGemm);
  if (rc) return rc;
  if (regs.empty()) return NRG_OK;
  std::vector<nrg::SpecTask> tasks;
  const int64_t chunk = 4096;
  for (size_t r = 0; r < regs.size(); r++) {
    const int64_t nt = (int64_t)(regs[r].i1 - regs[r].i0) * (regs[r].j1 - regs[r].j0);
    for (int64_t t0 = 0; t0 < nt; t0 += chunk) {
      nrg::SpecTask k{};
      k.t0 = t0;
      k.t1 = std::min(nt, t0 + chunk);
      k.region = (int)r;
      tasks.push_back(k);
    }
  }
  std::vector<char> img;
  const size_t ro = push(img, regs), to = push(img, tasks);
  rc = stage_desc(c, img, s);
  if (rc) return rc;
  nrg::MatsParams mp{};
  mp.mats = mats;
  mp.bosonic = prm->sign == 1 ? 1 : 0;
  mp.T = prm->T;
  const char* base = static_cast<const char*>(c->desc);
  nrg::PhaseScope ps(c, nrg::kPhSpecBin, s);
  CK(nrg::spec_mats_launch(reinterpret_cast<const nrg::SpecTask*>(base + to), (int)tasks.size(),
                           reinterpret_cast<const nrg::SpecRegion*>(base + ro), mp, re, im, s));
  return NRG_OK;
}

}  // extern "C"
