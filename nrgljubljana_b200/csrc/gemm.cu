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
// output, double-buffered in shared memory by asynchronous copies (cp.async).
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace nrg {
namespace {

constexpr int BM = kGemmBM, BN = kGemmBN, BK = kGemmBK, NT = kGemmThreads;
constexpr int PAD = 4;
constexpr int LDS = BM + PAD;  // shared-memory row stride (doubles) of both operand tiles

// Asynchronous 8-byte copy global -> shared (cp.async, no register staging); with ok false the
// destination is zero-filled and nothing is read (src must still be a valid address).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int sz = ok ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Copy the BK x BM slice of op(A) and the BK x BN slice of op(B) starting at k0 into the
// stage's shared-memory tiles As[k][m], Bs[k][n] (zeros outside the matrices). Consecutive
// threads read consecutive addresses of the contiguous direction of each operand.
__device__ __forceinline__ void issue_stage(const GemmSeg& g, int M, int N, int m0, int n0, int k0, double* As,
                                            double* Bs) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int e = tid + NT * i;
    int m, k;
    if (!g.transA) { k = e & (BK - 1); m = e >> 4; } else { m = e & (BM - 1); k = e >> 6; }
    const int gm = m0 + m, gk = k0 + k;
    const bool ok = gm < M && gk < g.K;
    const double* src = ok ? (g.transA ? g.A + (int64_t)gk * g.lda + gm : g.A + (int64_t)gm * g.lda + gk) : g.A;
    cp_async8(As + k * LDS + m, src, ok);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int e = tid + NT * i;
    int n, k;
    if (!g.transB) { n = e & (BN - 1); k = e >> 6; } else { k = e & (BK - 1); n = e >> 4; }
    const int gn = n0 + n, gk = k0 + k;
    const bool ok = gn < N && gk < g.K;
    const double* src = ok ? (g.transB ? g.B + (int64_t)gn * g.ldb + gk : g.B + (int64_t)gk * g.ldb + gn) : g.B;
    cp_async8(Bs + k * LDS + n, src, ok);
  }
  cp_async_commit();
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

  // The accumulators start from beta*C: the loads of C go out beside the first operand loads
  // instead of after the last product, which matters for the short-K updates (K = 128 of the
  // back-transform), where one exposed load latency is a large part of a tile's time.
  double acc[4][4][2];
  const bool addc = o.beta != 0.0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + wm + i * 8 + fr;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = n0 + wn + j * 8 + 2 * fc + h;
        acc[i][j][h] = (addc && r < o.M && c < o.N) ? o.beta * o.C[(int64_t)r * o.ldc + c] : 0.0;
      }
  }

  // Flatten (segment, k-chunk) into one sequence of steps.
  int total = 0;
  for (int s = 0; s < o.nseg; s++) total += (segs[o.seg0 + s].K + BK - 1) / BK;

  if (total > 0) {
    // Two stages: the copy of chunk step+1 runs while chunk step is multiplied. One barrier per
    // chunk: after it chunk step has landed for every thread and every thread has finished
    // reading the other stage (chunk step-1), which the next copy overwrites.
    int cs = 0, ck = 0;  // segment and k offset of the newest chunk issued
    while (segs[o.seg0 + cs].K <= 0) cs++;
    GemmSeg g = segs[o.seg0 + cs];
    issue_stage(g, o.M, o.N, m0, n0, 0, As[0], Bs[0]);
    double alpha_next = g.alpha;
    for (int step = 0; step < total; step++) {
      cp_async_wait_all();
      __syncthreads();
      const int buf = step & 1;
      const double alpha = alpha_next;
      if (step + 1 < total) {
        ck += BK;
        if (ck >= g.K) {
          cs++;
          while (segs[o.seg0 + cs].K <= 0) cs++;
          ck = 0;
          g = segs[o.seg0 + cs];
        }
        issue_stage(g, o.M, o.N, m0, n0, ck, As[buf ^ 1], Bs[buf ^ 1]);
        alpha_next = g.alpha;
      }
      const double* as = As[buf];
      const double* bs = Bs[buf];
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; i++) a[i] = as[(kk + fc) * LDS + wm + i * 8 + fr] * alpha;
#pragma unroll
        for (int j = 0; j < 4; j++) b[j] = bs[(kk + fc) * LDS + wn + j * 8 + fr];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) dmma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
  }

  // Epilogue: C = acc (= beta*C + the products).
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + wm + i * 8 + fr;
    if (r >= o.M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = n0 + wn + j * 8 + 2 * fc + h;
        if (c < o.N) o.C[(int64_t)r * o.ldc + c] = acc[i][j][h];
      }
    }
  }
}

__global__ void __launch_bounds__(NT, 5) gemm_batch_kernel(const GemmOut* __restrict__ outs,
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
__global__ void __launch_bounds__(NT, 5) gemm_one_kernel(const __grid_constant__ GemmOut o,
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
