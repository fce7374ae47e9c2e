// gemm.cu -- batched, segmented FP64 GEMM on the FP64 tensor cores (DMMA m8n8k4).
//
// Used for every GEMM-shaped step of the NRG step core: the recalculation leaves
// product / transform / rotate (numerics_ublas.hpp:108-140 of the reference), the
// prod_fit products of the spectral algorithms, the divide-and-conquer merges and the
// Householder back-transform of the eigensolver. tcgen05.mma has no f64 kind on sm_100a,
// so FP64 tensor work goes through mma.sync DMMA.
//
// One CTA (4 warps) computes a 64 x 64 tile of one output; each warp owns a 32 x 32
// sub-tile (4 x 4 DMMA tiles). K is walked in chunks of 16 over all segments of the
// output, double-buffered through registers into shared memory.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace nrg {
namespace {

constexpr int BM = kGemmBM, BN = kGemmBN, BK = kGemmBK, NT = kGemmThreads;
constexpr int PAD = 4;
constexpr int LDS = BM + PAD;  // shared-memory row stride (doubles) of both operand tiles

struct Stage {
  double a[8];
  double b[8];
};

// Load the BK x BM slice of op(A) and the BK x BN slice of op(B) starting at k0 into regs.
__device__ __forceinline__ void load_stage(Stage& s, const GemmSeg& g, int M, int N, int m0, int n0, int k0) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int e = tid + NT * i;
    int m, k;
    if (!g.transA) { k = e & (BK - 1); m = e >> 4; } else { m = e & (BM - 1); k = e >> 6; }
    const int gm = m0 + m, gk = k0 + k;
    double v = 0.0;
    if (gm < M && gk < g.K) v = g.transA ? g.A[(int64_t)gk * g.lda + gm] : g.A[(int64_t)gm * g.lda + gk];
    s.a[i] = v * g.alpha;
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int e = tid + NT * i;
    int n, k;
    if (!g.transB) { n = e & (BN - 1); k = e >> 6; } else { k = e & (BK - 1); n = e >> 4; }
    const int gn = n0 + n, gk = k0 + k;
    double v = 0.0;
    if (gn < N && gk < g.K) v = g.transB ? g.B[(int64_t)gn * g.ldb + gk] : g.B[(int64_t)gk * g.ldb + gn];
    s.b[i] = v;
  }
}

__device__ __forceinline__ void store_stage(const Stage& s, const GemmSeg& g, double* As, double* Bs) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int e = tid + NT * i;
    int m, k;
    if (!g.transA) { k = e & (BK - 1); m = e >> 4; } else { m = e & (BM - 1); k = e >> 6; }
    As[k * LDS + m] = s.a[i];
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int e = tid + NT * i;
    int n, k;
    if (!g.transB) { n = e & (BN - 1); k = e >> 6; } else { k = e & (BK - 1); n = e >> 4; }
    Bs[k * LDS + n] = s.b[i];
  }
}

// One 64 x 64 output tile `tt` (row-major tile order) of output o, whose segments are
// segs[o.seg0 .. o.seg0 + o.nseg).
__device__ __forceinline__ void gemm_tile(const GemmOut& o, const GemmSeg* __restrict__ segs, int tt) {
  __shared__ __align__(16) double As[2][BK * LDS];
  __shared__ __align__(16) double Bs[2][BK * LDS];
  const int tiles_n = (o.N + BN - 1) / BN;
  const int m0 = (tt / tiles_n) * BM, n0 = (tt % tiles_n) * BN;
  if (m0 >= o.M) return;  // outputs whose row count is set on the device may shrink

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int fr = lane >> 2, fc = lane & 3;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

  // Flatten (segment, k-chunk) into one sequence of steps.
  int total = 0;
  for (int s = 0; s < o.nseg; s++) total += (segs[o.seg0 + s].K + BK - 1) / BK;

  if (total > 0) {
    int cs = 0, ck = 0;  // current segment, k offset inside it
    while (segs[o.seg0 + cs].K <= 0) cs++;
    GemmSeg g = segs[o.seg0 + cs];
    Stage st;
    load_stage(st, g, o.M, o.N, m0, n0, 0);
    store_stage(st, g, As[0], Bs[0]);
    __syncthreads();
    int buf = 0;
    for (int step = 0; step < total; step++) {
      // advance to the next chunk and prefetch it into registers
      int ns = cs, nk = ck + BK;
      GemmSeg gn = g;
      const bool has_next = step + 1 < total;
      if (has_next) {
        if (nk >= g.K) {
          ns = cs + 1;
          while (segs[o.seg0 + ns].K <= 0) ns++;
          nk = 0;
          gn = segs[o.seg0 + ns];
        }
        load_stage(st, gn, o.M, o.N, m0, n0, nk);
      }
      const double* as = As[buf];
      const double* bs = Bs[buf];
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = as[(kk + fc) * LDS + wm + i * 8 + fr];
#pragma unroll
        for (int j = 0; j < 4; j++) b[j] = bs[(kk + fc) * LDS + wn + j * 8 + fr];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) dmma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
      if (has_next) {
        store_stage(st, gn, As[buf ^ 1], Bs[buf ^ 1]);
        cs = ns;
        ck = nk;
        g = gn;
      }
      __syncthreads();
      buf ^= 1;
    }
  }

  // Epilogue: C = beta*C + acc.
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + wm + i * 8 + fr;
    if (r >= o.M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = n0 + wn + j * 8 + 2 * fc + h;
        if (c < o.N) {
          double* p = o.C + (int64_t)r * o.ldc + c;
          *p = (o.beta == 0.0) ? acc[i][j][h] : fma(o.beta, *p, acc[i][j][h]);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(NT) gemm_batch_kernel(const GemmOut* __restrict__ outs,
                                                         const GemmSeg* __restrict__ segs, int nout) {
  // Locate the output that owns this tile (binary search over tile0).
  const int t = blockIdx.x;
  int lo = 0, hi = nout - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (outs[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const GemmOut o = outs[lo];
  gemm_tile(o, segs, t - o.tile0);
}

// Single output with a single segment, both passed by value (no descriptor memory).
__global__ void __launch_bounds__(NT) gemm_one_kernel(const __grid_constant__ GemmOut o,
                                                       const __grid_constant__ GemmSeg g) {
  gemm_tile(o, &g, blockIdx.x);
}

// Element e of the batch belongs to the last term whose off <= e; one product per element.
__global__ void __launch_bounds__(256) row_scale_kernel(const RowScale* __restrict__ terms, int nterm,
                                                        int64_t total) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nterm - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (terms[mid].off <= e) lo = mid; else hi = mid - 1;
    }
    const RowScale& r = terms[lo];
    const int64_t q = e - r.off;
    const int k = (int)(q / r.cols), c = (int)(q % r.cols);
    const double b = r.transB ? r.B[(int64_t)c * r.ldb + k] : r.B[(int64_t)k * r.ldb + c];
    r.T[q] = r.d[k] * b;
  }
}

}  // namespace

cudaError_t row_scale_launch(const RowScale* d_terms, int nterm, int64_t total, cudaStream_t stream) {
  if (nterm <= 0 || total <= 0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 16);
  row_scale_kernel<<<(unsigned)blocks, 256, 0, stream>>>(d_terms, nterm, total);
  return cudaGetLastError();
}

cudaError_t gemm_one_launch(const GemmOut& o, const GemmSeg& g, cudaStream_t stream) {
  const int tiles = ((o.M + BM - 1) / BM) * ((o.N + BN - 1) / BN);
  if (tiles <= 0) return cudaSuccess;
  GemmOut oo = o;
  oo.seg0 = 0;
  oo.nseg = 1;
  oo.tile0 = 0;
  gemm_one_kernel<<<tiles, NT, 0, stream>>>(oo, g);
  return cudaGetLastError();
}

cudaError_t gemm_batch_launch(const GemmOut* d_outs, const GemmSeg* d_segs, int nout, int ntiles,
                              cudaStream_t stream) {
  if (nout <= 0 || ntiles <= 0) return cudaSuccess;
  gemm_batch_kernel<<<ntiles, NT, 0, stream>>>(d_outs, d_segs, nout);
  return cudaGetLastError();
}

}  // namespace nrg
