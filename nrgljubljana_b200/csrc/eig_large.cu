// eig_large.cu -- batched FP64 symmetric eigensolver for blocks larger than kSmallMaxN.
//
// Replaces LAPACK dsyev/dsyevd as called by diagonalise() (c++/diag.hpp:62-115, 261-292
// of the reference) for the large symmetry blocks of an NRG step, with the output layout
// of copy_results (ascending eigenvalues, eigenvectors as rows, c++/diag.hpp:41-58).
//
// Pipeline per chunk of blocks (all blocks of the chunk advance together):
//   1. tridiag_kernel     one CTA per block: blocked Householder reduction A = Q T Q^T
//                         (panel width NB); the symmetric matrix-vector product streams
//                         the lower triangle from HBM once per column, the panel update
//                         is a rank-2NB update of the trailing lower triangle.
//   2. divide and conquer on T: leaves (<= kLeaf) by implicit QL in shared memory, merges
//      by rank-one tearing (Cuppen), deflation (small z and close poles with Givens
//      rotations), secular-equation roots with a two-pole rational model safeguarded by
//      bisection, Gu-Eisenstat recomputation of z for orthogonal vectors, and the merge
//      products as FP64 tensor-core GEMMs that skip the zero blocks of the children.
//   3. sort of the eigenvalues and row permutation of the eigenvectors.
//   4. back-transform with the compact-WY form of Q, panels of NBT reflectors, as GEMMs.
// Eigenvectors are kept as ROWS throughout (Zt = Z^T), the layout of the output.
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <vector>

#include "common.cuh"
#include "band.h"
#include "eig_large.h"
#include "eig_small.cuh"

namespace nrg {
namespace {

constexpr int kTriThreads = 128;
constexpr int NB = 16;     // tridiagonalisation panel width
constexpr int NBT = 128;   // back-transform panel width
constexpr int kLeaf = 32;  // divide-and-conquer leaves have at most this order
constexpr int kMaxLargeN = 10240;  // the tridiagonalisation's shared memory (68 KB + 16 n bytes) fits to here
// Merge nodes whose prep arrays exceed this many bytes keep them in global scratch (kPrepGlobalB
// bytes per row of the block) instead of shared memory.
constexpr size_t kPrepSmemMax = 200 * 1024;
constexpr size_t kPrepGlobalB = 80;

struct LargeBlock {
  double* H;      // input (consumed); then the eigenvector rows of T during divide and
                  // conquer; then the VT factors of the back-transform
  double* evals;
  double* evecs;  // output; scratch for the merge matrices during divide and conquer
  double* W1;     // n x ldp: packed lower triangle being reduced; Householder vectors after
  double* W2;     // n x n: panel W of the reduction; grouped rows of a merge; back-transform W
  double* d;
  double* e;
  double* tau;
  double* lam;    // eigenvalues of the current divide-and-conquer nodes
  double* dsort;  // per node: non-deflated poles, ascending
  double* dgrp;   // per node: non-deflated poles, grouped order
  double* zgrp;   // per node: z in grouped order
  double* GT;     // per back-transform panel of nb reflectors: Gram matrix V^T V then T (nb x nb each)
  int* rank;      // per node: sorted position of grouped entry
  int* perm;      // final eigenvalue order
  char* pscr;     // kPrepGlobalB bytes per row: merge-prep arrays of nodes too large for shared memory
  int* info;
  int n, npanel;
  int ldp, pad_;  // leading dimension of the packed lower triangle in W1 (multiple of 32)
};

struct DcLeaf {
  int blk, a0, a1, pad;
};

struct DcNode {
  int blk, a, m, b;
  int gout;  // index of the first of its two GEMM outputs in the level's GEMM arrays
  int pad;
};

struct DcState {
  int K, k1, k2, k3;
  double rho;
};

// ---------------------------------------------------------------- tridiagonalisation

// Column sums of an 8-column slab: lane l holds x[c] = A(i_l, j0+c) * v[i_l]; returns, in
// every lane, the sum over all 32 lanes of x[c] for c = (l >> 2) & 7 (9 shuffles).
NRG_DEV double slab_colsum8(double (&x)[8], int lane) {
  {
    const bool up = (lane & 16) != 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const double send = up ? x[q] : x[q + 4];
      const double keep = up ? x[q + 4] : x[q];
      x[q] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
  }
  {
    const bool up = (lane & 8) != 0;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const double send = up ? x[q] : x[q + 2];
      const double keep = up ? x[q + 2] : x[q];
      x[q] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
  }
  {
    const bool up = (lane & 4) != 0;
    const double send = up ? x[0] : x[1];
    const double keep = up ? x[1] : x[0];
    x[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  x[0] += __shfl_xor_sync(0xffffffffu, x[0], 2);
  x[0] += __shfl_xor_sync(0xffffffffu, x[0], 1);
  return x[0];
}

// ---- bulk asynchronous copies (TMA, non-multicast) into the CTA's own shared memory
NRG_DEV unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

NRG_DEV void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

NRG_DEV void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Orders this thread's earlier generic-proxy global writes before later bulk (async-proxy)
// reads of the same memory.
NRG_DEV void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

NRG_DEV void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Acquire a tensor map that lives in global memory and was written by a host copy: orders the
// copy's generic-proxy writes before this thread's tensormap-proxy reads of the 128-byte map,
// so that no descriptor cached from an earlier map at the same address is used. The maps are
// rewritten at the same addresses for every chunk of blocks and every call.
NRG_DEV void tmap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(map) : "memory");
}

// Bounded wait for phase `parity` of an mbarrier; false if the bound ran out.
NRG_DEV bool mbar_wait(uint64_t* bar, unsigned parity, int bound = (1 << 26)) {
  const unsigned a = smem_u32(bar);
  for (int it = 0; it < bound; it++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 2-D bulk tensor copy (TMA, non-multicast) of one box at coordinates (x, y) into this
// CTA's shared memory, completing on an mbarrier.
NRG_DEV void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// The same with an L2 eviction-priority hint (an access policy from createpolicy): the slabs of
// a trailing triangle that is streamed once per column and does not fit in L2 go first, so
// that the panel's vectors (read three times per column) stay.
NRG_DEV void tma_load_2d_hint(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, "
      "%3}], [%4], %5;" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

NRG_DEV uint64_t l2_evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Loads and stores of the panel's vectors (V and W columns, re-read three times per column of
// the panel) with an evict-last L2 hint, so that the streamed slabs do not push them out.
NRG_DEV uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
NRG_DEV double ld_keep(const double* a, uint64_t pol) {
  double v;
  asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}
NRG_DEV void st_keep(double* a, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}

constexpr int kStages = 4;                 // slabs in flight per warp
constexpr int kSlabRows = 64;              // rows of a slab (two per lane)
constexpr int kSlabD = kSlabRows * 8;      // doubles per slab: 64 rows x 8 columns
constexpr int kTriWarps = kTriThreads / 32;

// y[i] += sum_{j >= s0} A(i, j) v[j] for s0 <= i < n. A is the packed lower triangle
// (A(i, j) = P[j*ld + i] for i >= j, zero above the diagonal and in the padding) behind the
// 2-D tensor map `tmap` (inner extent ld rows, outer extent n columns, box 64 x 8). The
// triangle is cut into 64-row x 8-column slabs; the slabs, in tile-row order, are split
// evenly between the warps, and each warp streams its slabs through a ring of kStages
// shared-memory buffers, one TMA box copy per slab completing on the buffer's mbarrier.
// A lane owns rows l and l+32 of the slab: row sums stay in registers until the tile row
// changes, column sums are transposed across the warp; both are added to y (shared memory).
// `parity` holds the warp's mbarrier phase bits across calls.
// gwarp / gnwarps: this warp's index among the warps that share the product (the warps of
// one CTA, or of every CTA of a cluster), and their number; y receives this warp's part.
template <int STAGES = kStages, bool EVICT_FIRST = false>
NRG_DEV void symv_lower(const CUtensorMap* tmap, int n, int s0, const double* v, double* y, double* ring,
                        uint64_t* bars, unsigned& parity, int* err, int gwarp, int gnwarps) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int T0 = s0 >> 6, Tn = (n - 1) >> 6, sl0 = s0 >> 3, slmax = (n - 1) >> 3;
  auto rowlen = [&](int I) { return min(8 * I + 7, slmax) - sl0 + 1; };
  long long S = 0;
  for (int I = T0; I <= Tn; I++) S += rowlen(I);
  const long long f0 = S * gwarp / gnwarps, f1 = S * (gwarp + 1) / gnwarps;
  if (f0 >= f1) return;
  double* myring = ring + (size_t)warp * STAGES * kSlabD;
  uint64_t* mybar = bars + warp * STAGES;
  auto advance = [&](int& I_, int& sl_) {
    if (sl_ < min(8 * I_ + 7, slmax)) {
      sl_++;
    } else {
      I_++;
      sl_ = sl0;
    }
  };
  const uint64_t policy = EVICT_FIRST ? l2_evict_first_policy() : 0;
  auto issue = [&](int I_, int sl_, int st) {
    if (lane == 0) {
      mbar_expect_tx(mybar + st, (unsigned)(kSlabD * sizeof(double)));
      if (EVICT_FIRST)
        tma_load_2d_hint(myring + st * kSlabD, tmap, I_ * kSlabRows, sl_ * 8, mybar + st, policy);
      else
        tma_load_2d(myring + st * kSlabD, tmap, I_ * kSlabRows, sl_ * 8, mybar + st);
    }
  };
  int I = T0;
  long long acc = 0;
  while (acc + rowlen(I) <= f0) {
    acc += rowlen(I);
    I++;
  }
  int sl = sl0 + (int)(f0 - acc);
  int pI = I, psl = sl;
  const int npre = (int)((f1 - f0) < (long long)STAGES ? (f1 - f0) : (long long)STAGES);
  for (int t = 0; t < npre; t++) {
    issue(pI, psl, t);
    advance(pI, psl);
  }
  double r0 = 0.0, r1 = 0.0;
  int cI = I, csl = sl;
  for (long long f = f0; f < f1; f++) {
    const int st = (int)((f - f0) % STAGES);
    if (!mbar_wait(mybar + st, (parity >> st) & 1u)) {
      // a copy never completed: flag the block, wait (bounded) for the copies still in
      // flight so that none lands after this call, and stop streaming
      if (lane == 0) atomicExch(err, -5);
      const long long last = (f + STAGES < f1) ? f + STAGES : f1;
      for (long long g = f + 1; g < last; g++) {
        const int sg = (int)((g - f0) % STAGES);
        mbar_wait(mybar + sg, (parity >> sg) & 1u, 1 << 22);
        parity ^= 1u << sg;
      }
      parity ^= 1u << st;
      return;
    }
    parity ^= 1u << st;
    const double* buf = myring + st * kSlabD;
    const int ia = cI * kSlabRows + lane, ib = ia + 32, j0 = csl << 3;
    const double va = (ia >= s0 && ia < n) ? v[ia] : 0.0;
    const double vb = (ib >= s0 && ib < n) ? v[ib] : 0.0;
    double cp[8];
    if (j0 >= s0 && j0 + 8 <= cI * kSlabRows && j0 + 8 <= n) {
      // strictly left of the tile row's diagonal and inside the trailing block: no masks
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const double a0 = buf[c * kSlabRows + lane], a1 = buf[c * kSlabRows + 32 + lane];
        const double vj = v[j0 + c];
        r0 = fma(a0, vj, r0);
        r1 = fma(a1, vj, r1);
        cp[c] = fma(a0, va, a1 * vb);
      }
    } else {
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int jj = j0 + c;
        const bool cok = jj >= s0 && jj < n;  // reduced columns hold Householder vectors
        const double a0 = cok ? buf[c * kSlabRows + lane] : 0.0;
        const double a1 = cok ? buf[c * kSlabRows + 32 + lane] : 0.0;
        const double vj = cok ? v[jj] : 0.0;
        r0 = fma(a0, vj, r0);
        r1 = fma(a1, vj, r1);
        cp[c] = (jj < ia ? a0 * va : 0.0) + (jj < ib ? a1 * vb : 0.0);  // diagonal: row sum only
      }
    }
    __syncwarp();
    if (f + STAGES < f1) {  // refill this stage with the slab STAGES ahead
      issue(pI, psl, st);
      advance(pI, psl);
    }
    const double cs = slab_colsum8(cp, lane);
    const int jc = j0 + ((lane >> 2) & 7);
    if ((lane & 3) == 0 && jc >= s0 && jc < n && cs != 0.0) atomicAdd(&y[jc], cs);
    int nI = cI, nsl = csl;
    advance(nI, nsl);
    if (f + 1 == f1 || nI != cI) {
      if (ia >= s0 && ia < n && r0 != 0.0) atomicAdd(&y[ia], r0);
      if (ib >= s0 && ib < n && r1 != 0.0) atomicAdd(&y[ib], r1);
      r0 = r1 = 0.0;
    }
    cI = nI;
    csl = nsl;
  }
}

// A(i, j) -= sum_{q < nbp} V(i,q) W(j,q) + W(i,q) V(j,q) for s0 <= j <= i < n, with
// V(i, q) = P[(p0+q)*ld + i] and W(i, q) = W[q*n + i], on the FP64 tensor cores:
// A -= Y X^T with Y = [V | W] (rows i) and X = [W | V] (rows j), K = 2NB. A warp owns a
// 32 x 32 tile (rows i, columns j) as 4 x 4 DMMA 8x8x4 accumulators whose rows run along
// the contiguous direction of P, so every load and store of the tile and of the operands
// is 8 consecutive doubles per quarter-warp. The row operands Y of a tile row stay in
// registers while the warp walks the columns. The tiles of the trailing lower triangle,
// in tile-row order, are split evenly between the warps.
// CG: read P and W past the L1 cache (ld.global.cg); needed when other CTAs wrote them,
// since an SM's L1 may still hold lines it read before those writes.
template <bool CG>
NRG_DEV double ldp(const double* p) {
  if constexpr (CG) return __ldcg(p);
  else return *p;
}

template <bool CG>
NRG_DEV void panel_update(double* __restrict__ P, const double* __restrict__ W, int n, int ld, int p0, int nbp,
                          int s0, int gwarp, int gnwarps) {
  const int lane = threadIdx.x & 31;
  const int r = lane >> 2, c4 = lane & 3;
  const int T0 = s0 >> 5, Tn = (n - 1) >> 5;
  const int nt = Tn - T0 + 1;
  const long long S = (long long)nt * (nt + 1) / 2;
  const long long f0 = S * gwarp / gnwarps, f1 = S * (gwarp + 1) / gnwarps;
  if (f0 >= f1) return;
  int I = T0;
  long long acc0 = 0;
  while (acc0 + (I - T0 + 1) <= f0) {
    acc0 += I - T0 + 1;
    I++;
  }
  int J = T0 + (int)(f0 - acc0);
  double ya[4][2 * NB / 4];  // A fragments of Y for the current tile row
  int rowI = -1;
  for (long long f = f0; f < f1; f++) {
    const int i0 = I << 5, j0 = J << 5;
    if (rowI != I) {
      rowI = I;
#pragma unroll
      for (int ks = 0; ks < 2 * NB / 4; ks++) {
        const int q = 4 * ks + c4;
        const bool first = q < NB;
        const int qq = first ? q : q - NB;
        const double* row = first ? P + (size_t)(p0 + qq) * ld : W + (size_t)qq * n;
#pragma unroll
        for (int mi = 0; mi < 4; mi++) {
          const int ii = i0 + 8 * mi + r;
          ya[mi][ks] = (qq < nbp && ii < n) ? -ldp<CG>(row + ii) : 0.0;
        }
      }
    }
    double acc[4][4][2];
#pragma unroll
    for (int mi = 0; mi < 4; mi++)
#pragma unroll
      for (int ni = 0; ni < 4; ni++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int ii = i0 + 8 * mi + r, jj = j0 + 8 * ni + 2 * c4 + h;
          const bool ok = jj >= s0 && ii < n && ii >= jj;
          acc[mi][ni][h] = ok ? ldp<CG>(P + (size_t)jj * ld + ii) : 0.0;
        }
#pragma unroll
    for (int ks = 0; ks < 2 * NB / 4; ks++) {
      const int q = 4 * ks + c4;
      const bool first = q < NB;
      const int qq = first ? q : q - NB;
      const double* row = first ? W + (size_t)qq * n : P + (size_t)(p0 + qq) * ld;
      double b[4];
#pragma unroll
      for (int ni = 0; ni < 4; ni++) {
        const int jj = j0 + 8 * ni + r;
        b[ni] = (qq < nbp && jj < n) ? ldp<CG>(row + jj) : 0.0;
      }
#pragma unroll
      for (int mi = 0; mi < 4; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) dmma884(acc[mi][ni][0], acc[mi][ni][1], ya[mi][ks], b[ni]);
    }
#pragma unroll
    for (int mi = 0; mi < 4; mi++)
#pragma unroll
      for (int ni = 0; ni < 4; ni++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int ii = i0 + 8 * mi + r, jj = j0 + 8 * ni + 2 * c4 + h;
          if (jj >= s0 && ii < n && ii >= jj) P[(size_t)jj * ld + ii] = acc[mi][ni][h];
        }
    if (J < I) {
      J++;
    } else {
      I++;
      J = T0;
    }
  }
}

// Packs the upper triangle of the row-major input (the lower triangle in column terms)
// into W1 with leading dimension ldp: W1[j*ldp + i] = H[j*n + i] for i >= j, zero for i < j
// and in the padding rows n <= i < ldp. Grid (row chunks of 8, blocks).
__global__ void __launch_bounds__(256) pack_lower_kernel(const LargeBlock* __restrict__ blocks) {
  const LargeBlock B = blocks[blockIdx.y];
  const int n = B.n, ld = B.ldp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = blockIdx.x * 8 + warp;
  if (j >= n) return;
  const double* src = B.H + (size_t)j * n;
  double* dst = B.W1 + (size_t)j * ld;
  for (int i = lane; i < ld; i += 32) dst[i] = (i >= j && i < n) ? src[i] : 0.0;
}

// One CTA per block: blocked (NB) Householder reduction of the packed lower triangle in W1
// (leading dimension ldp) to tridiagonal form; d, e, tau out; Householder vector k is left
// in column k (W1[k*ldp + k+1 ..], with a unit at k+1).
// STAGES slabs in flight per warp; MINB CTAs per SM for the register budget: <4, 2> (two per
// SM, 255 registers) and <2, 3> (three per SM, 168 registers and a smaller ring).
template <int STAGES, int MINB>
__global__ void __launch_bounds__(kTriThreads, MINB) tridiag_kernel(const LargeBlock* __restrict__ blocks,
                                                                    const CUtensorMap* __restrict__ tmaps) {
  extern __shared__ __align__(16) double sm[];
  __shared__ __align__(8) uint64_t bars[kTriWarps * STAGES];
  const LargeBlock B = blocks[blockIdx.x];
  const int n = B.n, ld = B.ldp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  double* A = B.W1;
  double* W = B.W2;
  const uint64_t keep = l2_evict_last_policy();
  // TMA destinations: 1024-byte aligned ring of STAGES slabs per warp
  double* ring = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(sm) + 1023) & ~(uintptr_t)1023);
  double* v = ring + kTriWarps * STAGES * kSlabD;      // n
  double* y = v + n;                                   // n
  double* part = y + n;                                // nwarps * 2NB
  double* cwv = part + nwarps * 2 * NB;                // 2NB
  double* red = cwv + 2 * NB;                          // 64 (two halves for block_sum_1b)
  int phase = 0;
  unsigned parity = 0;
  if (lane == 0) {
    for (int st = 0; st < STAGES; st++) mbar_init(bars + warp * STAGES + st, 1);
    fence_mbar_init();
    tmap_acquire(tmaps + blockIdx.x);  // lane 0 issues this warp's bulk copies
  }
  __syncthreads();

  for (int p0 = 0; p0 < n - 2; p0 += NB) {
    const int pe = min(p0 + NB, n - 2);
    for (int k = p0; k < pe; k++) {
      const int j = k - p0;
      // (1) current column k (rows k..n-1) = stored column minus the pending panel terms
      {
        double wk[NB], vk[NB];
#pragma unroll
        for (int q = 0; q < NB; q++) {
          wk[q] = (q < j) ? W[(size_t)q * n + k] : 0.0;
          vk[q] = (q < j) ? A[(size_t)(p0 + q) * ld + k] : 0.0;
        }
        for (int i = k + tid; i < n; i += nt) {
          double a = A[(size_t)k * ld + i];
#pragma unroll
          for (int q = 0; q < NB; q++)
            if (q < j) a -= ld_keep(A + (size_t)(p0 + q) * ld + i, keep) * wk[q] + ld_keep(W + (size_t)q * n + i, keep) * vk[q];
          v[i] = a;
          y[i] = 0.0;
        }
      }
      __syncthreads();
      // (2) Householder reflector for rows k+1..n-1 (dlarfg convention, v[k+1] = 1)
      double ps = 0.0;
      for (int i = k + 2 + tid; i < n; i += nt) ps += v[i] * v[i];
      // alpha is read before the barrier inside block_sum_1b: thread 0 overwrites v[k+1] with
      // the unit below, with no barrier between, and a warp that read it late would scale its
      // part of the reflector with a wrong beta (and disagree with the others on tau)
      const double alpha = v[k + 1];
      const double sigma = block_sum_1b(ps, red, phase);
      double tau = 0.0, beta = alpha, scale = 1.0;
      if (sigma > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
        tau = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
      }
      if (tid == 0) {
        B.d[k] = v[k];
        B.e[k] = beta;
        B.tau[k] = tau;
      }
      for (int i = k + 2 + tid; i < n; i += nt) {
        const double vi = v[i] * scale;
        v[i] = vi;
        st_keep(A + (size_t)k * ld + i, vi, keep);
      }
      // column k of W1 now holds v_k below the diagonal; clear its entries above, inside
      // the back-transform panel, so that the panel's V block is exactly unit lower trapezoidal
      const int kb0 = (k / NBT) * NBT;
      for (int i = kb0 + 1 + tid; i <= k; i += nt) A[(size_t)k * ld + i] = 0.0;
      if (tid == 0) {
        v[k + 1] = 1.0;
        A[(size_t)k * ld + k + 1] = 1.0;
      }
      __syncthreads();
      if (tau != 0.0) {
        // (3) y = A_panel_start(k+1:, k+1:) v - V (W^T v) - W (V^T v), W[:, j] = tau y - K v
        symv_lower<STAGES, true>(tmaps + blockIdx.x, n, k + 1, v, y, ring, bars, parity, B.info, warp, nwarps);
        if (j > 0) {
          double pw[NB], pv[NB];
#pragma unroll
          for (int q = 0; q < NB; q++) pw[q] = pv[q] = 0.0;
          for (int i = k + 1 + tid; i < n; i += nt) {
            const double vi = v[i];
#pragma unroll
            for (int q = 0; q < NB; q++)
              if (q < j) {
                pw[q] = fma(ld_keep(W + (size_t)q * n + i, keep), vi, pw[q]);
                pv[q] = fma(ld_keep(A + (size_t)(p0 + q) * ld + i, keep), vi, pv[q]);
              }
          }
#pragma unroll
          for (int q = 0; q < NB; q++) {
            if (q < j) {
              const double a = warp_sum(pw[q]);
              const double b = warp_sum(pv[q]);
              if (lane == 0) {
                part[warp * 2 * NB + q] = a;
                part[warp * 2 * NB + NB + q] = b;
              }
            }
          }
          __syncthreads();
          if (tid < 2 * NB) {
            double s = 0.0;
            for (int w = 0; w < nwarps; w++) s += part[w * 2 * NB + tid];
            cwv[tid] = s;
          }
        }
        __syncthreads();
        double cw[NB], cv[NB];
#pragma unroll
        for (int q = 0; q < NB; q++) {
          cw[q] = (q < j) ? cwv[q] : 0.0;
          cv[q] = (q < j) ? cwv[NB + q] : 0.0;
        }
        double pp = 0.0;
        for (int i = k + 1 + tid; i < n; i += nt) {
          double yi = y[i];
#pragma unroll
          for (int q = 0; q < NB; q++)
            if (q < j) yi -= ld_keep(A + (size_t)(p0 + q) * ld + i, keep) * cw[q] + ld_keep(W + (size_t)q * n + i, keep) * cv[q];
          yi *= tau;
          y[i] = yi;
          pp = fma(yi, v[i], pp);
        }
        const double Kc = 0.5 * tau * block_sum_1b(pp, red, phase);
        for (int i = k + 1 + tid; i < n; i += nt) st_keep(W + (size_t)j * n + i, y[i] - Kc * v[i], keep);
      } else {
        for (int i = k + 1 + tid; i < n; i += nt) W[(size_t)j * n + i] = 0.0;
      }
      __syncthreads();
    }
    panel_update<false>(A, W, n, ld, p0, pe - p0, pe, warp, nwarps);
    fence_proxy_async_global();  // the next symv reads the updated trailing block by bulk copies
    __syncthreads();
  }
  if (tid == 0) {
    B.d[n - 2] = A[(size_t)(n - 2) * ld + n - 2];
    B.e[n - 2] = A[(size_t)(n - 2) * ld + n - 1];
    B.d[n - 1] = A[(size_t)(n - 1) * ld + n - 1];
    B.e[n - 1] = 0.0;
    B.tau[n - 2] = 0.0;
    B.tau[n - 1] = 0.0;
  }
  __syncthreads();
  int bad = 0;
  for (int i = tid; i < n; i += nt) bad |= !(isfinite(B.d[i]) && isfinite(B.e[i]));
  if (__syncthreads_or(bad) && tid == 0) atomicMin(B.info, -2);
}

// ---------------------------------------------------------------- large blocks, few of them
// One thread-block cluster per block: the blocked reduction of tridiag_kernel with the TMA
// slabs of A v and the tiles of the panel update split over the warps of every CTA of the
// cluster. The column work (current column, reflector) is repeated by every CTA on its own
// copy of the vectors; each CTA writes its slice of rows to global memory. The parts of A v
// and of the dot products are summed through distributed shared memory: after the first
// barrier each CTA reduces its slice of rows, after the second the scalar y^T v is summed;
// the third makes the column of W visible to the cluster, a fourth follows each panel update.
// Every CTA executes the same sequence of barriers whatever the data.
constexpr int kTclC = 8;  // CTAs per cluster (16 when the blocks are few)

template <int STAGES>
__global__ void __launch_bounds__(kTriThreads, 1) tridiag_tcl_kernel(const LargeBlock* __restrict__ blocks,
                                                                     const CUtensorMap* __restrict__ tmaps) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) double sm[];
  __shared__ __align__(8) uint64_t bars[kTriWarps * STAGES];
  const int C = (int)cl.num_blocks(), rk = (int)cl.block_rank();
  const int bi = blockIdx.x / C;
  const LargeBlock B = blocks[bi];
  const int n = B.n, ld = B.ldp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  const int gw = rk * nwarps + warp, gnw = C * nwarps;
  double* A = B.W1;
  double* W = B.W2;
  // The arrays that other CTAs read (y, dots, pps) sit at fixed offsets from the start of the
  // dynamic shared memory, so that map_shared_rank finds them at the same offsets in every
  // CTA; the 1024-byte aligned TMA ring comes last (its padding depends on where the CTA's
  // shared memory window starts, which differs between CTAs sharing an SM).
  double* y = sm;                                   // n: this CTA's part of A v; its slice: the reduced y
  double* dots = y + n;                             // 2NB: this CTA's part of W^T v, V^T v
  double* pps = dots + 2 * NB;                      // 2: this CTA's part of y^T v
  double* v = pps + 2;                              // n: current column, then the reflector
  double* part = v + n;                             // nwarps * 2NB
  double* cwv = part + nwarps * 2 * NB;             // 2NB: the sums
  double* red = cwv + 2 * NB;                       // 64 (two halves for block_sum_1b)
  double* ring = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(red + 64) + 1023) & ~(uintptr_t)1023);
  int phase = 0;
  unsigned parity = 0;
  if (lane == 0) {
    for (int st = 0; st < STAGES; st++) mbar_init(bars + warp * STAGES + st, 1);
    fence_mbar_init();
    tmap_acquire(tmaps + bi);  // lane 0 issues this warp's bulk copies
  }
  __syncthreads();

  for (int p0 = 0; p0 < n - 2; p0 += NB) {
    const int pe = min(p0 + NB, n - 2);
    for (int k = p0; k < pe; k++) {
      const int j = k - p0;
      // (1) current column k (rows k..n-1) = stored column minus the pending panel terms
      {
        double wk[NB], vk[NB];
#pragma unroll
        for (int q = 0; q < NB; q++) {
          wk[q] = (q < j) ? __ldcg(W + (size_t)q * n + k) : 0.0;
          vk[q] = (q < j) ? __ldcg(A + (size_t)(p0 + q) * ld + k) : 0.0;
        }
        for (int i = k + tid; i < n; i += nt) {
          double a = __ldcg(A + (size_t)k * ld + i);
#pragma unroll
          for (int q = 0; q < NB; q++)
            if (q < j) a -= __ldcg(A + (size_t)(p0 + q) * ld + i) * wk[q] + __ldcg(W + (size_t)q * n + i) * vk[q];
          v[i] = a;
          y[i] = 0.0;
        }
      }
      __syncthreads();
      // (2) Householder reflector for rows k+1..n-1 (dlarfg convention, v[k+1] = 1)
      double ps = 0.0;
      for (int i = k + 2 + tid; i < n; i += nt) ps += v[i] * v[i];
      const double alpha = v[k + 1];  // before the barrier: thread 0 sets v[k+1] = 1 below
      const double sigma = block_sum_1b(ps, red, phase);
      double tau = 0.0, beta = alpha, scale = 1.0;
      if (sigma > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
        tau = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
      }
      if (rk == 0 && tid == 0) {
        B.d[k] = v[k];
        B.e[k] = beta;
        B.tau[k] = tau;
      }
      for (int i = k + 2 + tid; i < n; i += nt) v[i] *= scale;
      if (tid == 0) v[k + 1] = 1.0;
      __syncthreads();
      // column k of A is written back only in (5): other CTAs may still be reading it in (1)
      // (3) this CTA's part of A v and of the dot products W^T v, V^T v over its slice of rows
      const int ch1 = (n - k - 1 + C - 1) / C, lo1 = k + 1 + rk * ch1, hi1 = min(n, lo1 + ch1);
      if (tau != 0.0) symv_lower<STAGES>(tmaps + bi, n, k + 1, v, y, ring, bars, parity, B.info, gw, gnw);
      {
        double pw[NB], pv[NB];
#pragma unroll
        for (int q = 0; q < NB; q++) pw[q] = pv[q] = 0.0;
        if (tau != 0.0 && j > 0) {
          for (int i = lo1 + tid; i < hi1; i += nt) {
            const double vi = v[i];
#pragma unroll
            for (int q = 0; q < NB; q++)
              if (q < j) {
                pw[q] = fma(__ldcg(W + (size_t)q * n + i), vi, pw[q]);
                pv[q] = fma(__ldcg(A + (size_t)(p0 + q) * ld + i), vi, pv[q]);
              }
          }
        }
#pragma unroll
        for (int q = 0; q < NB; q++) {
          const double a = warp_sum(pw[q]);
          const double b = warp_sum(pv[q]);
          if (lane == 0) {
            part[warp * 2 * NB + q] = a;
            part[warp * 2 * NB + NB + q] = b;
          }
        }
        __syncthreads();
        if (tid < 2 * NB) {
          double t = 0.0;
          for (int w = 0; w < nwarps; w++) t += part[w * 2 * NB + tid];
          dots[tid] = t;
        }
      }
      cl.sync();  // (B1) the parts of A v and of the dot products are complete
      // (4) this CTA's slice: y = (sum of the parts - V (W^T v) - W (V^T v)) tau
      if (tid < 2 * NB) {
        double t = 0.0;
        for (int q = 0; q < C; q++) t += cl.map_shared_rank(dots, q)[tid];
        cwv[tid] = t;
      }
      __syncthreads();
      double pp = 0.0;
      if (tau != 0.0) {
        double cw[NB], cv[NB];
#pragma unroll
        for (int q = 0; q < NB; q++) {
          cw[q] = (q < j) ? cwv[q] : 0.0;
          cv[q] = (q < j) ? cwv[NB + q] : 0.0;
        }
        for (int i = lo1 + tid; i < hi1; i += nt) {
          double yi = 0.0;
          for (int q = 0; q < C; q++) yi += cl.map_shared_rank(y, q)[i];
#pragma unroll
          for (int q = 0; q < NB; q++)
            if (q < j) yi -= __ldcg(A + (size_t)(p0 + q) * ld + i) * cw[q] + __ldcg(W + (size_t)q * n + i) * cv[q];
          yi *= tau;
          pp = fma(yi, v[i], pp);
          y[i] = yi;  // only this CTA's slice is read from here on, and only by this CTA
        }
      }
      const double ppb = block_sum_1b(pp, red, phase);
      if (tid == 0) pps[0] = ppb;
      cl.sync();  // (B2) every CTA has its slice of y and its part of y^T v
      double yv = 0.0;
      for (int q = 0; q < C; q++) yv += cl.map_shared_rank(pps, q)[0];
      const double Kc = 0.5 * tau * yv;
      for (int i = lo1 + tid; i < hi1; i += nt) {
        W[(size_t)j * n + i] = (tau != 0.0) ? y[i] - Kc * v[i] : 0.0;
        A[(size_t)k * ld + i] = v[i];  // the reflector, unit at k+1
      }
      if (rk == 0) {  // zeros from the start of its back-transform panel down to the diagonal
        const int kb0 = (k / NBT) * NBT;
        for (int i = kb0 + 1 + tid; i <= k; i += nt) A[(size_t)k * ld + i] = 0.0;
      }
      cl.sync();  // (B3) column j of W and column k of the reflectors are visible to the cluster
    }
    panel_update<true>(A, W, n, ld, p0, pe - p0, pe, gw, gnw);
    fence_proxy_async_global();  // the next products read the updated trailing block by bulk copies
    cl.sync();                   // (B4)
    fence_proxy_async_global();
  }
  if (rk == 0) {
    if (tid == 0) {
      B.d[n - 2] = __ldcg(A + (size_t)(n - 2) * ld + n - 2);
      B.e[n - 2] = __ldcg(A + (size_t)(n - 2) * ld + n - 1);
      B.d[n - 1] = __ldcg(A + (size_t)(n - 1) * ld + n - 1);
      B.e[n - 1] = 0.0;
      B.tau[n - 2] = 0.0;
      B.tau[n - 1] = 0.0;
    }
    __syncthreads();
    int bad = 0;
    for (int i = tid; i < n; i += nt) bad |= !(isfinite(B.d[i]) && isfinite(B.e[i]));
    if (__syncthreads_or(bad) && tid == 0) atomicMin(B.info, -2);
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------- mid-size tridiagonalisation
// Blocks with small_max_n < n <= mid_max_n (nrg_tuning): the whole lower triangle fits in shared memory,
// packed by columns (column j holds rows j..n-1 at pcol(j)), so the unblocked Householder
// reduction runs without touching HBM or L2 after the first read of H. Output as
// tridiag_kernel: d, e, tau, and v_k in row k of W1 (unit at k+1, zeros from the start of
// its back-transform panel up to k).
constexpr int kMidThreads = 512;

NRG_DEV int pcol(int j, int n) { return j * n - (j * (j - 1)) / 2; }

__global__ void __launch_bounds__(kMidThreads) tridiag_smem_kernel(const LargeBlock* __restrict__ blocks) {
  extern __shared__ __align__(16) double sm[];
  const LargeBlock B = blocks[blockIdx.x];
  const int n = B.n, ld = B.ldp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  const int tot = n * (n + 1) / 2;
  double* P = sm;
  double* v = P + tot;
  double* w = v + n;
  double* red = w + n;  // 64 (two halves for block_sum_1b)
  int phase = 0;
  // column j of the lower triangle is row j of H from the diagonal on (row-major upper)
  for (int j = warp; j < n; j += nwarps) {
    const double* src = B.H + (size_t)j * n;
    double* dst = P + pcol(j, n) - j;
    for (int i = j + lane; i < n; i += 32) dst[i] = src[i];
  }
  __syncthreads();
  double* A = B.W1;
  for (int k = 0; k < n - 2; k++) {
    const int ck = pcol(k, n) - k;  // P[ck + i] = A(i, k), i >= k
    double ps = 0.0;
    for (int i = k + 2 + tid; i < n; i += nt) {
      const double x = P[ck + i];
      ps = fma(x, x, ps);
    }
    const double sigma = block_sum_1b(ps, red, phase);
    const double alpha = P[ck + k + 1];
    double tau = 0.0, beta = alpha, scale = 1.0;
    if (sigma > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
      tau = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    for (int i = k + 1 + tid; i < n; i += nt) {
      const double vi = (i == k + 1) ? 1.0 : P[ck + i] * scale;
      v[i] = vi;
      A[(size_t)k * ld + i] = vi;
    }
    const int kb0 = (k / NBT) * NBT;
    for (int i = kb0 + 1 + tid; i <= k; i += nt) A[(size_t)k * ld + i] = 0.0;
    if (tid == 0) {
      B.d[k] = P[ck + k];
      B.e[k] = beta;
      B.tau[k] = tau;
    }
    __syncthreads();
    if (tau == 0.0) continue;  // uniform: every thread computed the same sigma
    // w = tau * A22 v over rows/columns k+1..n-1; thread i reads row i left of the
    // diagonal and column i from the diagonal down: n-k-1 entries for every i
    for (int i = k + 1 + tid; i < n; i += nt) {
      double s0 = 0.0, s1 = 0.0;
      int addr = pcol(k + 1, n) + (i - (k + 1));  // A(i, k+1)
      for (int c = k + 1; c < i; c++) {
        s0 = fma(P[addr], v[c], s0);
        addr += n - c - 1;
      }
      const int ci = pcol(i, n) - i;
      for (int r = i; r < n; r++) s1 = fma(P[ci + r], v[r], s1);
      w[i] = tau * (s0 + s1);
    }
    __syncthreads();
    double pp = 0.0;
    for (int i = k + 1 + tid; i < n; i += nt) pp = fma(w[i], v[i], pp);
    const double Kc = 0.5 * tau * block_sum_1b(pp, red, phase);
    for (int i = k + 1 + tid; i < n; i += nt) w[i] -= Kc * v[i];
    __syncthreads();
    // rank-2 update of the trailing triangle, contiguous from pcol(k+1) to the end
    {
      int j = k + 1, off = tid;
      while (j < n && off >= n - j) {
        off -= n - j;
        j++;
      }
      int p = pcol(k + 1, n) + tid;
      while (j < n) {
        const int i = j + off;
        P[p] -= v[i] * w[j] + w[i] * v[j];
        p += nt;
        off += nt;
        while (j < n && off >= n - j) {
          off -= n - j;
          j++;
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    const int c2 = pcol(n - 2, n);
    B.d[n - 2] = P[c2];
    B.e[n - 2] = P[c2 + 1];
    B.d[n - 1] = P[pcol(n - 1, n)];
    B.e[n - 1] = 0.0;
    B.tau[n - 2] = 0.0;
    B.tau[n - 1] = 0.0;
  }
  __syncthreads();
  int bad = 0;
  for (int i = tid; i < n; i += nt) bad |= !(isfinite(B.d[i]) && isfinite(B.e[i]));
  if (__syncthreads_or(bad) && tid == 0) atomicMin(B.info, -2);
}

// ---------------------------------------------------------------- cluster tridiagonalisation
// Blocks with mid_max_n < n <= cluster_max_n (nrg_tuning): the packed lower triangle is spread over the
// shared memory of a thread-block cluster of C CTAs (column j lives in CTA j mod C) and the
// unblocked Householder reduction runs there; the CTAs read each other's shared memory
// (distributed shared memory, plain loads, no bulk copies). Two cluster barriers per column:
//   A  column k is final in its owner, and every CTA has finished reading the partial
//      products of the previous column;
//      every CTA reads column k from its owner and builds the same reflector v itself; each
//      CTA forms its share of A v: per row, the part left of the diagonal from its own
//      columns; per owned column (one warp), the part from the diagonal down;
//   B  every CTA sums the shares of all CTAs for every row in a fixed order (so all CTAs
//      hold the same w) and updates its own columns.
// Output as tridiag_kernel.
constexpr int kClThreads = 512;

// Offset of owned column t (global column j = r + t*C) in the local storage of CTA r.
__host__ __device__ inline long long cl_loff(int t, int r, int C, int n) {
  return (long long)t * (n - r) - (long long)C * t * (t - 1) / 2;
}

// Doubles of shared memory a CTA of a C-cluster needs for a block of order n.
__host__ __device__ inline long long cl_smem_doubles(int n, int C) {
  const int T0 = (n + C - 1) / C;  // columns of CTA 0, the largest share
  return ((cl_loff(T0, 0, C, n) + 1) & ~1LL) + 4LL * n + 64;
}

__global__ void __launch_bounds__(kClThreads) tridiag_cluster_kernel(const LargeBlock* __restrict__ blocks,
                                                                     int lmax) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks(), r = (int)cl.block_rank();
  const LargeBlock B = blocks[blockIdx.x / C];
  extern __shared__ __align__(16) double sm[];
  const int n = B.n, ld = B.ldp, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  double* Pl = sm;          // owned columns, packed
  double* v = Pl + lmax;    // n
  double* w = v + n;        // n
  double* yp = w + n;       // n: row part of this CTA's share of A v
  double* yc = yp + n;      // n: column part (entries of owned columns)
  double* red = yc + n;     // 64 (two halves for block_sum_1b)
  int phase = 0;
  const int T = (n - r + C - 1) / C;
  for (int t = warp; t < T; t += nwarps) {
    const int j = r + t * C;
    const double* src = B.H + (size_t)j * n;
    double* dst = Pl + cl_loff(t, r, C, n) - j;
    for (int i = j + lane; i < n; i += 32) dst[i] = src[i];
  }
  double* A = B.W1;
  for (int k = 0; k < n - 2; k++) {
    cl.sync();  // A
    const int o = k % C;
    // column k from its owner: colr[i] = A(i, k)
    const double* colr = cl.map_shared_rank(Pl + cl_loff(k / C, o, C, n) - k, o);
    double ps = 0.0;
    for (int i = k + 2 + tid; i < n; i += nt) {
      const double x = colr[i];
      ps = fma(x, x, ps);
    }
    const double sigma = block_sum_1b(ps, red, phase);
    const double alpha = colr[k + 1];
    double tau = 0.0, beta = alpha, scale = 1.0;
    if (sigma > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
      tau = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    for (int i = k + 1 + tid; i < n; i += nt) {
      const double vi = (i == k + 1) ? 1.0 : colr[i] * scale;
      v[i] = vi;
      if (r == o) A[(size_t)k * ld + i] = vi;
    }
    if (r == o) {
      const int kb0 = (k / NBT) * NBT;
      for (int i = kb0 + 1 + tid; i <= k; i += nt) A[(size_t)k * ld + i] = 0.0;
      if (tid == 0) {
        B.d[k] = colr[k];
        B.e[k] = beta;
        B.tau[k] = tau;
      }
    }
    __syncthreads();
    if (tau == 0.0) continue;  // the same in every CTA
    // this CTA's share of A v over rows/columns k+1..n-1
    const int t0 = (k + 1 - r > 0) ? (k + 1 - r + C - 1) / C : 0;  // first owned column >= k+1
    for (int i = k + 1 + tid; i < n; i += nt) {
      double s = 0.0;
      long long addr = cl_loff(t0, r, C, n) - (r + t0 * C) + i;  // A(i, c) for c = r + t0*C
      for (int t = t0, c = r + t0 * C; c < i; t++, c += C) {
        s = fma(Pl[addr], v[c], s);
        addr += (n - r - (long long)t * C) - C;
      }
      yp[i] = s;
    }
    for (int t = t0 + warp; t < T; t += nwarps) {
      const int j = r + t * C;
      const double* col = Pl + cl_loff(t, r, C, n) - j;
      double dot = 0.0;
      for (int i = j + lane; i < n; i += 32) dot = fma(col[i], v[i], dot);
      dot = warp_sum(dot);
      if (lane == 0) yc[j] = dot;
    }
    cl.sync();  // B
    double pd = 0.0;
    for (int i = k + 1 + tid; i < n; i += nt) {
      double y = 0.0;
      for (int q = 0; q < C; q++) y += cl.map_shared_rank(yp, q)[i];
      y += cl.map_shared_rank(yc, i % C)[i];
      const double wi = tau * y;
      w[i] = wi;
      pd = fma(wi, v[i], pd);
    }
    const double Kc = 0.5 * tau * block_sum_1b(pd, red, phase);  // its barrier also publishes w
    // rank-2 update of the owned trailing columns with w' = w - Kc v
    {
      int t = t0, off = tid;
      while (t < T && off >= n - (r + t * C)) {
        off -= n - (r + t * C);
        t++;
      }
      long long p = cl_loff(t0, r, C, n) + tid;
      while (t < T) {
        const int j = r + t * C, i = j + off;
        const double wj = w[j] - Kc * v[j], wi = w[i] - Kc * v[i];
        Pl[p] -= v[i] * wj + wi * v[j];
        p += nt;
        off += nt;
        while (t < T && off >= n - (r + t * C)) {
          off -= n - (r + t * C);
          t++;
        }
      }
    }
  }
  if (tid == 0) {
    if (r == (n - 2) % C) {
      const double* col = Pl + cl_loff((n - 2) / C, r, C, n) - (n - 2);
      B.d[n - 2] = col[n - 2];
      B.e[n - 2] = col[n - 1];
      B.tau[n - 2] = 0.0;
    }
    if (r == (n - 1) % C) {
      const double* col = Pl + cl_loff((n - 1) / C, r, C, n) - (n - 1);
      B.d[n - 1] = col[n - 1];
      B.e[n - 1] = 0.0;
      B.tau[n - 1] = 0.0;
    }
  }
  cl.sync();  // the last remote reads are done; d and e are complete
  if (r == 0) {
    int bad = 0;
    for (int i = tid; i < n; i += nt) bad |= !(isfinite(B.d[i]) && isfinite(B.e[i]));
    if (__syncthreads_or(bad) && tid == 0) atomicMin(B.info, -2);
  }
}

// ---------------------------------------------------------------- divide and conquer: leaves
__global__ void __launch_bounds__(128) dc_leaf_kernel(const LargeBlock* __restrict__ blocks,
                                                      const DcLeaf* __restrict__ leaves) {
  __shared__ double Z[kLeaf * (kLeaf + 1)];
  __shared__ double d[kLeaf], e[kLeaf], C[2 * kLeaf], S[2 * kLeaf];
  __shared__ int ctl[8];
  const DcLeaf L = leaves[blockIdx.x];
  const LargeBlock B = blocks[L.blk];
  const int n = B.n, a0 = L.a0, nl = L.a1 - L.a0, ld = kLeaf + 1, tid = threadIdx.x;
  for (int i = tid; i < nl; i += blockDim.x) {
    double di = B.d[a0 + i];
    if (i == 0 && a0 > 0) di -= fabs(B.e[a0 - 1]);             // rank-one tearing at the left cut
    if (i == nl - 1 && L.a1 < n) di -= fabs(B.e[L.a1 - 1]);    // and at the right cut
    d[i] = di;
    e[i] = (i < nl - 1) ? B.e[a0 + i] : 0.0;
  }
  for (int idx = tid; idx < nl * nl; idx += blockDim.x) {
    const int r = idx / nl, c = idx % nl;
    Z[r * ld + c] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int st = smem_ql(d, e, nl, Z, ld, nl, C, S, ctl);
  if (st && tid == 0) atomicMax(B.info, st);
  for (int r = tid; r < nl; r += blockDim.x) B.lam[a0 + r] = d[r];
  for (int idx = tid; idx < nl * nl; idx += blockDim.x) {
    const int r = idx / nl, c = idx % nl;  // row r of Zt = column r of Z
    B.H[(size_t)(a0 + r) * n + a0 + c] = Z[c * ld + r];
  }
}

// ---------------------------------------------------------------- divide and conquer: merge prep
// Shared-memory layout for a node of order N (P = next power of two >= N).
struct PrepLayout {
  size_t key, sidx, zs, lst, rcs, rpos, fl, total;
};

__host__ __device__ inline size_t r16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline PrepLayout prep_layout(int N) {
  int P = 1;
  while (P < N) P <<= 1;
  PrepLayout L;
  size_t o = 0;
  L.key = o;  o += r16(sizeof(double) * (size_t)P);   // pole values, sorted
  L.sidx = o; o += r16(sizeof(int) * (size_t)P);      // original position
  L.zs = o;   o += r16(sizeof(double) * (size_t)N);   // z in sorted order
  L.lst = o;  o += r16(sizeof(int) * (size_t)N);      // non-deflated from the front, deflated from the back
  L.rcs = o;  o += r16(sizeof(double2) * (size_t)N);  // rotation (c, s)
  L.rpos = o; o += r16(sizeof(int2) * (size_t)N);     // rotation (pos_p, pos_j), later: grouped slot
  L.fl = o;   o += r16((size_t)N);                    // support flags per sorted position
  L.total = o;
  return L;
}

__global__ void __launch_bounds__(512) dc_prep_kernel(const LargeBlock* __restrict__ blocks,
                                                      const DcNode* __restrict__ nodes, DcState* __restrict__ states,
                                                      GemmOut* __restrict__ gouts, GemmSeg* __restrict__ gsegs,
                                                      size_t smem_bytes) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[32];
  __shared__ int cnt[8];
  const DcNode nd = nodes[blockIdx.x];
  const LargeBlock B = blocks[nd.blk];
  const int n = B.n, a = nd.a, m = nd.m, b = nd.b, N = b - a;
  const int tid = threadIdx.x, nt = blockDim.x;
  int P = 1;
  while (P < N) P <<= 1;
  const PrepLayout PL = prep_layout(N);
  // a node whose arrays do not fit the shared memory of the launch uses its rows' slice of the
  // block's global scratch (nodes of one level cover disjoint rows)
  char* smc = PL.total <= smem_bytes ? reinterpret_cast<char*>(sm) : B.pscr + kPrepGlobalB * (size_t)a;
  double* key = reinterpret_cast<double*>(smc + PL.key);
  int* sidx = reinterpret_cast<int*>(smc + PL.sidx);
  double* zs = reinterpret_cast<double*>(smc + PL.zs);
  int* lst = reinterpret_cast<int*>(smc + PL.lst);
  double2* rcs = reinterpret_cast<double2*>(smc + PL.rcs);
  int2* rpos = reinterpret_cast<int2*>(smc + PL.rpos);
  unsigned char* fl = reinterpret_cast<unsigned char*>(smc + PL.fl);
  double* Z = B.H;
  double* G = B.W2;

  // 1. clear the off-diagonal child blocks of the node
  const int n1 = m - a, n2 = b - m;
  for (int idx = tid; idx < n1 * n2; idx += nt) {
    const int r = idx / n2, c = idx % n2;
    Z[(size_t)(a + r) * n + m + c] = 0.0;
    const int r2 = idx / n1, c2 = idx % n1;
    Z[(size_t)(m + r2) * n + a + c2] = 0.0;
  }
  // 2. poles and the rank-one vector z = [last row of child 1; sign(beta) first row of child 2] / sqrt(2)
  const double beta = B.e[m - 1];
  const double rho = 2.0 * fabs(beta);
  const double sg = beta >= 0.0 ? 1.0 : -1.0;
  for (int s = tid; s < P; s += nt) {
    key[s] = (s < N) ? B.lam[a + s] : INFINITY;
    sidx[s] = s;
  }
  __syncthreads();
  // 3. bitonic sort (key, sidx) ascending
  for (int k = 2; k <= P; k <<= 1) {
    for (int jb = k >> 1; jb > 0; jb >>= 1) {
      for (int i = tid; i < P; i += nt) {
        const int ixj = i ^ jb;
        if (ixj > i) {
          const bool asc = (i & k) == 0;
          const double ki = key[i], kj = key[ixj];
          const bool sw = asc ? (ki > kj || (ki == kj && sidx[i] > sidx[ixj])) : (ki < kj || (ki == kj && sidx[i] < sidx[ixj]));
          if (sw) {
            key[i] = kj;
            key[ixj] = ki;
            const int t = sidx[i];
            sidx[i] = sidx[ixj];
            sidx[ixj] = t;
          }
        }
      }
      __syncthreads();
    }
  }
  // A non-finite pole (the block was already flagged) could move a padding slot forward:
  // leave such a node untouched rather than index outside it.
  int badidx = 0;
  for (int s = tid; s < N; s += nt) badidx |= (sidx[s] >= N);
  if (__syncthreads_or(badidx)) {
    if (tid == 0) atomicMin(B.info, -3);
    return;
  }
  double dmx = 0.0, zmx = 0.0;
  for (int s = tid; s < N; s += nt) {
    const int c = a + sidx[s];
    const double z = (c < m ? Z[(size_t)c * n + (m - 1)] : sg * Z[(size_t)c * n + m]) * 0.70710678118654752440;
    zs[s] = z;
    fl[s] = (c < m) ? 1 : 2;
    dmx = fmax(dmx, fabs(key[s]));
    zmx = fmax(zmx, fabs(z));
  }
  dmx = block_max(dmx, red);
  zmx = block_max(zmx, red);
  // 4. deflation scan (serial)
  if (tid == 0) {
    const double tol = 8.0 * kEps * fmax(dmx, zmx);
    int K = 0, nd_ = 0, nrot = 0;
    if (rho * zmx <= tol) {
      for (int s = 0; s < N; s++) lst[N - 1 - (nd_++)] = s;
    } else {
      int p = -1;
      for (int s = 0; s < N; s++) {
        if (rho * fabs(zs[s]) <= tol) {
          lst[N - 1 - (nd_++)] = s;
          continue;
        }
        if (p < 0) {
          p = s;
          continue;
        }
        const double zp = zs[p], zj = zs[s];
        const double t = hypot(zp, zj);
        const double c = zj / t, sn = zp / t;
        if (fabs((key[s] - key[p]) * c * sn) <= tol) {
          // rotate rows (p, s): z_p -> 0, z_s -> t; p deflates
          rcs[nrot] = make_double2(c, sn);
          rpos[nrot] = make_int2(p, s);
          nrot++;
          const double dp = key[p], ds = key[s];
          key[p] = c * c * dp + sn * sn * ds;
          key[s] = sn * sn * dp + c * c * ds;
          zs[s] = t;
          zs[p] = 0.0;
          fl[s] |= fl[p];
          fl[p] |= fl[s];
          lst[N - 1 - (nd_++)] = p;
          p = s;
        } else {
          lst[K++] = p;
          p = s;
        }
      }
      if (p >= 0) lst[K++] = p;
    }
    cnt[0] = K;
    cnt[1] = nd_;
    cnt[2] = nrot;
  }
  __syncthreads();
  const int K = cnt[0], ndefl = cnt[1], nrot = cnt[2];
  // 5. apply the deflation rotations to the eigenvector rows, in order
  for (int r = 0; r < nrot; r++) {
    const double c = rcs[r].x, sn = rcs[r].y;
    const size_t rp = (size_t)(a + sidx[rpos[r].x]) * n, rj = (size_t)(a + sidx[rpos[r].y]) * n;
    for (int col = a + tid; col < b; col += nt) {
      const double zp = Z[rp + col], zj = Z[rj + col];
      Z[rp + col] = c * zp - sn * zj;
      Z[rj + col] = sn * zp + c * zj;
    }
    __syncthreads();
  }
  // 6. group the non-deflated entries by support: child 1 only, both, child 2 only
  if (tid == 0) {
    int k1 = 0, k2 = 0, k3 = 0;
    for (int t = 0; t < K; t++) {
      const int f = fl[lst[t]];
      if (f == 1) k1++;
      else if (f == 3) k2++;
      else k3++;
    }
    int g1 = 0, g2 = k1, g3 = k1 + k2;
    for (int t = 0; t < K; t++) {
      const int s = lst[t];
      const int f = fl[s];
      const int g = (f == 1) ? g1++ : (f == 3) ? g2++ : g3++;
      B.rank[a + g] = t;
      B.dgrp[a + g] = key[s];
      B.zgrp[a + g] = zs[s];
      B.dsort[a + t] = key[s];
      // remember where the row goes: reuse rpos.x as the grouped slot of sorted position s
      rpos[s].x = g;
    }
    for (int q = 0; q < ndefl; q++) {
      const int s = lst[N - 1 - q];
      B.lam[a + K + q] = key[s];
      rpos[s].x = K + q;
    }
    cnt[3] = k1;
    cnt[4] = k2;
    cnt[5] = k3;
    DcState st;
    st.K = K;
    st.k1 = k1;
    st.k2 = k2;
    st.k3 = k3;
    st.rho = rho;
    states[blockIdx.x] = st;
    // the two merge GEMMs: rows of child-1 columns from types 1+2, child-2 columns from 2+3
    gouts[nd.gout].M = K;
    gouts[nd.gout + 1].M = K;
    gsegs[nd.gout].K = k1 + k2;
    gsegs[nd.gout + 1].K = k2 + k3;
    gsegs[nd.gout + 1].A = B.evecs + (size_t)a * n + a + k1;
    gsegs[nd.gout + 1].B = B.W2 + (size_t)(a + k1) * n + m;
  }
  __syncthreads();
  // 7. copy the rows into grouped order in G (non-deflated first, then deflated)
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  for (int s = warp; s < N; s += nwarps) {
    const size_t src = (size_t)(a + sidx[s]) * n, dst = (size_t)(a + rpos[s].x) * n;
    for (int col = a + lane; col < b; col += 32) G[dst + col] = Z[src + col];
  }
}

// ---------------------------------------------------------------- divide and conquer: secular equation
// Root j of 1 + rho sum_i z_i^2 / (d_i - lambda) = 0 with poles d ascending. One warp per
// root, lanes over i. On exit Dt[j][g] = d_g - lambda_j for every grouped entry g.
__global__ void __launch_bounds__(256) dc_secular_kernel(const LargeBlock* __restrict__ blocks,
                                                         const DcNode* __restrict__ nodes,
                                                         const DcState* __restrict__ states) {
  const DcNode nd = nodes[blockIdx.x];
  const DcState st = states[blockIdx.x];
  const LargeBlock B = blocks[nd.blk];
  const int K = st.K;
  if (K == 0) return;
  const int n = B.n, a = nd.a;
  const double rho = st.rho;
  const int lane = threadIdx.x & 31;
  const int wg = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int wstride = gridDim.y * (blockDim.x >> 5);
  const double* ds = B.dsort + a;
  const double* dg = B.dgrp + a;
  const double* zg = B.zgrp + a;
  const int* rk = B.rank + a;
  double* Dt = B.evecs + (size_t)a * n + a;
  for (int j = wg; j < K; j += wstride) {
    double dorg, lo, hi, tau;
    int p1, p2;
    if (K == 1) {
      const double z = zg[0];
      if (lane == 0) {
        Dt[0] = -rho * z * z;
        B.lam[a] = ds[0] + rho * z * z;
      }
      continue;
    }
    if (j < K - 1) {
      const double dj = ds[j], mid = 0.5 * (ds[j + 1] - dj);
      double s = 0.0;
      for (int i = lane; i < K; i += 32) {
        const double z = zg[i];
        s += z * z / ((dg[i] - dj) - mid);
      }
      const double f = 1.0 + rho * warp_sum(s);
      if (f >= 0.0) {
        dorg = dj;
        lo = 0.0;
        hi = mid;
      } else {
        dorg = ds[j + 1];
        lo = -mid;
        hi = 0.0;
      }
      p1 = j;
      p2 = j + 1;
    } else {
      double s = 0.0;
      for (int i = lane; i < K; i += 32) s += zg[i] * zg[i];
      dorg = ds[K - 1];
      lo = 0.0;
      hi = rho * warp_sum(s);
      p1 = K - 2;
      p2 = K - 1;
    }
    tau = 0.5 * (lo + hi);
    const double d1 = ds[p1] - dorg, d2 = ds[p2] - dorg;
    for (int it = 0; it < 100; it++) {
      double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0;
      for (int i = lane; i < K; i += 32) {
        const double del = (dg[i] - dorg) - tau;
        const double t = zg[i] / del;
        if (rk[i] <= p1) {
          psi = fma(zg[i], t, psi);
          dpsi = fma(t, t, dpsi);
        } else {
          phi = fma(zg[i], t, phi);
          dphi = fma(t, t, dphi);
        }
      }
      psi = rho * warp_sum(psi);
      dpsi = rho * warp_sum(dpsi);
      phi = rho * warp_sum(phi);
      dphi = rho * warp_sum(dphi);
      const double f = 1.0 + psi + phi;
      const double err = 8.0 * (fabs(psi) + fabs(phi)) + 2.0 + 3.0 * fabs(tau) * (dpsi + dphi);
      if (fabs(f) <= kEps * err) break;
      if (f < 0.0) lo = tau; else hi = tau;
      // two-pole rational model through poles p1, p2 matching f and f'
      const double del1 = d1 - tau, del2 = d2 - tau;
      const double cc = f - del1 * dpsi - del2 * dphi;
      const double s1 = del1 * del1 * dpsi, s2 = del2 * del2 * dphi;
      const double A1 = cc * (del1 + del2) + s1 + s2;
      const double A0 = cc * del1 * del2 + s1 * del2 + s2 * del1;
      double eta;
      if (cc == 0.0) {
        eta = A0 / A1;
      } else {
        const double disc = sqrt(fabs(A1 * A1 - 4.0 * cc * A0));
        eta = (A1 <= 0.0) ? (A1 - disc) / (2.0 * cc) : 2.0 * A0 / (A1 + disc);
      }
      double tn = tau + eta;
      if (!(tn > lo && tn < hi)) tn = 0.5 * (lo + hi);
      if (tn == tau) break;
      tau = tn;
    }
    for (int i = lane; i < K; i += 32) Dt[(size_t)j * n + i] = (dg[i] - dorg) - tau;
    if (lane == 0) B.lam[a + j] = dorg + tau;
  }
}

// ---------------------------------------------------------------- divide and conquer: vectors
// z-hat by the Gu-Eisenstat product formula (into dgrp, free after the secular solve), then
// u_j(g) = zhat_g / (d_g - lambda_j), normalised, written over Dt in place (same grouped
// column order). Both kernels spread a node over gridDim.y CTAs.
__global__ void __launch_bounds__(256) dc_zhat_kernel(const LargeBlock* __restrict__ blocks,
                                                      const DcNode* __restrict__ nodes,
                                                      const DcState* __restrict__ states) {
  const DcNode nd = nodes[blockIdx.x];
  const DcState st = states[blockIdx.x];
  const LargeBlock B = blocks[nd.blk];
  const int K = st.K;
  const int n = B.n, a = nd.a;
  const double* ds = B.dsort + a;
  const double* zg = B.zgrp + a;
  const int* rk = B.rank + a;
  const double* Dt = B.evecs + (size_t)a * n + a;
  const double rho = st.rho;
  for (int g = blockIdx.y * blockDim.x + threadIdx.x; g < K; g += gridDim.y * blockDim.x) {
    const int i = rk[g];
    const double di = ds[i];
    double p0 = -Dt[(size_t)(K - 1) * n + g] / rho, p1 = 1.0;
    int j = 0;
    for (; j + 1 < i; j += 2) {  // two independent product chains
      p0 *= -Dt[(size_t)j * n + g] / (ds[j] - di);
      p1 *= -Dt[(size_t)(j + 1) * n + g] / (ds[j + 1] - di);
    }
    for (; j < i; j++) p0 *= -Dt[(size_t)j * n + g] / (ds[j] - di);
    for (; j + 1 < K - 1; j += 2) {
      p0 *= -Dt[(size_t)j * n + g] / (ds[j + 1] - di);
      p1 *= -Dt[(size_t)(j + 1) * n + g] / (ds[j + 2] - di);
    }
    for (; j < K - 1; j++) p0 *= -Dt[(size_t)j * n + g] / (ds[j + 1] - di);
    B.dgrp[a + g] = copysign(sqrt(fabs(p0 * p1)), zg[g]);
  }
}

__global__ void __launch_bounds__(256) dc_vectors_kernel(const LargeBlock* __restrict__ blocks,
                                                         const DcNode* __restrict__ nodes,
                                                         const DcState* __restrict__ states) {
  const DcNode nd = nodes[blockIdx.x];
  const DcState st = states[blockIdx.x];
  const LargeBlock B = blocks[nd.blk];
  const int K = st.K;
  const int n = B.n, a = nd.a, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int wg = blockIdx.y * (blockDim.x >> 5) + warp, wstride = gridDim.y * (blockDim.x >> 5);
  // deflated rows are final: grouped copy (W2) back to the node's rows a+K.. (H)
  for (int r = a + K + wg; r < nd.b; r += wstride)
    for (int col = a + lane; col < nd.b; col += 32) B.H[(size_t)r * n + col] = B.W2[(size_t)r * n + col];
  const double* zh = B.dgrp + a;
  double* Dt = B.evecs + (size_t)a * n + a;
  for (int j = wg; j < K; j += wstride) {
    double* row = Dt + (size_t)j * n;
    double ss = 0.0;
    for (int g = lane; g < K; g += 32) {
      const double u = zh[g] / row[g];
      ss = fma(u, u, ss);
    }
    const double inv = 1.0 / sqrt(warp_sum(ss));
    for (int g = lane; g < K; g += 32) row[g] = zh[g] / row[g] * inv;
  }
}

// ---------------------------------------------------------------- final order
__global__ void __launch_bounds__(1024) sort_final_kernel(const LargeBlock* __restrict__ blocks) {
  extern __shared__ __align__(16) double key[];
  const LargeBlock B = blocks[blockIdx.x];
  const int n = B.n, tid = threadIdx.x, nt = blockDim.x;
  int P = 1;
  while (P < n) P <<= 1;
  int* idx = reinterpret_cast<int*>(key + P);
  for (int s = tid; s < P; s += nt) {
    key[s] = (s < n) ? B.lam[s] : INFINITY;
    idx[s] = s;
  }
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1) {
    for (int jb = k >> 1; jb > 0; jb >>= 1) {
      for (int i = tid; i < P; i += nt) {
        const int ixj = i ^ jb;
        if (ixj > i) {
          const bool asc = (i & k) == 0;
          const double ki = key[i], kj = key[ixj];
          const bool sw = asc ? (ki > kj || (ki == kj && idx[i] > idx[ixj])) : (ki < kj || (ki == kj && idx[i] < idx[ixj]));
          if (sw) {
            key[i] = kj;
            key[ixj] = ki;
            const int t = idx[i];
            idx[i] = idx[ixj];
            idx[ixj] = t;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int s = tid; s < n; s += nt) {
    B.evals[s] = key[s];
    B.perm[s] = idx[s];
  }
}

// evecs[r][:] = W1[perm[r]][:]; grid (rows / 8, blocks)
__global__ void __launch_bounds__(256) permute_rows_kernel(const LargeBlock* __restrict__ blocks) {
  const LargeBlock B = blocks[blockIdx.y];
  const int n = B.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = blockIdx.x * 8 + warp;
  if (r >= n) return;
  int pr = B.perm[r];
  if (pr < 0 || pr >= n) pr = r;  // only after a flagged non-finite block
  const double* src = B.H + (size_t)pr * n;
  double* dst = B.evecs + (size_t)r * n;
  for (int c = lane; c < n; c += 32) dst[c] = src[c];
}

// ---------------------------------------------------------------- back-transform factors
// T of the compact-WY form H_k0 ... H_k0+nb-1 = I - V T V^T (forward, columnwise), from
// the Gram matrix G = V^T V (nb x nb) at GT + gt_off, written to GT + gt_off + nb^2.
struct PanelRef {
  int blk, k0, nb, pad;
  long long gt_off;
};

__global__ void __launch_bounds__(NBT) tfactor_kernel(const LargeBlock* __restrict__ blocks,
                                                      const PanelRef* __restrict__ panels) {
  extern __shared__ __align__(16) double tsm[];
  const PanelRef P = panels[blockIdx.x];
  const LargeBlock B = blocks[P.blk];
  const int nb = P.nb, t = threadIdx.x, lt = NBT + 1;
  double* Ts = tsm;           // NBT x (NBT+1)
  double* w = tsm + NBT * lt;  // NBT
  const double* G = B.GT + P.gt_off;
  double* T = B.GT + P.gt_off + (size_t)nb * nb;
  for (int r = 0; r < nb; r++) Ts[r * lt + t] = 0.0;
  __syncthreads();
  for (int q = 0; q < nb; q++) {
    const double tq = B.tau[P.k0 + q];
    // w = -tau_q G[0:q, q]; T[0:q, q] = T[0:q, 0:q] w
    if (t < q) w[t] = -tq * G[t * nb + q];
    __syncthreads();
    if (t < q) {
      double s = 0.0;
      for (int r = t; r < q; r++) s += Ts[t * lt + r] * w[r];
      Ts[t * lt + q] = s;
    }
    if (t == q) Ts[q * lt + q] = tq;
    __syncthreads();
  }
  if (t < nb)
    for (int r = 0; r < nb; r++) T[r * nb + t] = Ts[r * lt + t];
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

size_t large_block_doubles(int n, bool two_stage) {
  const size_t ldp = (size_t)(n + 31) / 32 * 32;
  return (size_t)n * ldp + (size_t)n * n + 8 * (size_t)n + 2 * (size_t)NBT * n + 2 * (size_t)n + 64 * 13 +
         (prep_layout(n).total > kPrepSmemMax ? (kPrepGlobalB * (size_t)n + 7) / 8 : 0) +
         (two_stage ? band_extra_doubles(n) + 4 * 64 : 0);
}

}  // namespace

int eig_large_run(nrg_ctx* c, const std::vector<int>& which, const int* n, double* const* H, double* const* evals,
                  double* const* evecs, int* info_dev, cudaStream_t s) {
  std::vector<int> ord(which);
  std::stable_sort(ord.begin(), ord.end(), [n](int x, int y) { return n[x] > n[y]; });
  const int mid_max_n = c->tune.mid_max_n, cluster_max_n = c->tune.cluster_max_n;
  // Two-stage reduction for the largest blocks when they are few (the first nts of `ord`).
  int nts_all = 0;
  if (c->tune.band_min_n > 0) {
    while (nts_all < (int)ord.size() && n[ord[nts_all]] >= c->tune.band_min_n) nts_all++;
    if (nts_all > c->tune.band_max_blocks) nts_all = 0;
  }
  for (int b : ord)
    if (n[b] > kMaxLargeN)
      return fail(NRG_ERR_ARG, "block %d: order %d exceeds the supported maximum %d", b, n[b], kMaxLargeN);
  // Chunk the blocks so that their workspaces fit in the context limit.
  const size_t limit = ws_available(c);  // chunks fit what the arena can grow to now
  size_t pos = 0;
  while (pos < ord.size()) {
    size_t bytes = 0, end = pos;
    while (end < ord.size()) {
      const size_t bb = align_up(sizeof(double) * large_block_doubles(n[ord[end]], (int)end < nts_all), 256);
      if (end > pos && bytes + bb > limit) break;
      bytes += bb;
      end++;
    }
    int rc = ensure_ws(c, bytes);
    if (rc) return rc;
    // ---- per-block descriptors
    std::vector<LargeBlock> blk;
    std::vector<BandBlock> bblk;  // the chunk's two-stage blocks (its first nts, the largest)
    std::vector<int> shift;       // row offset of each block's reflectors: 1, or kBand (two-stage)
    char* base = static_cast<char*>(c->ws);
    size_t off = 0;
    int maxn = 0, maxpanel = 0;
    const int nts = std::max(0, std::min((int)end, nts_all) - (int)pos);
    for (size_t t = pos; t < end; t++) {
      const int b = ord[t], nb_ = n[b];
      LargeBlock L{};
      auto take = [&](size_t nd) {
        double* p = reinterpret_cast<double*>(base + off);
        off += align_up(sizeof(double) * nd, 256);
        return p;
      };
      L.H = H[b];
      L.evals = evals[b];
      L.evecs = evecs[b];
      L.ldp = (nb_ + 31) / 32 * 32;
      L.W1 = take((size_t)nb_ * L.ldp);
      L.W2 = take((size_t)nb_ * nb_);
      L.d = take(nb_);
      L.e = take(nb_);
      L.tau = take(nb_);
      L.lam = take(nb_);
      L.dsort = take(nb_);
      L.dgrp = take(nb_);
      L.zgrp = take(nb_);
      L.npanel = (nb_ - 2 + NBT - 1) / NBT;
      L.GT = take(2 * (size_t)NBT * nb_);  // >= sum over panels of 2 nb^2
      int* ip = reinterpret_cast<int*>(take(nb_));
      L.rank = ip;
      L.perm = ip + nb_;
      L.pscr = prep_layout(nb_).total > kPrepSmemMax
                   ? reinterpret_cast<char*>(take((kPrepGlobalB * (size_t)nb_ + 7) / 8)) : nullptr;
      L.info = info_dev + b;
      L.n = nb_;
      if ((int)(t - pos) < nts) {
        // two-stage: reflectors of stage 1 at rows k, unit at k + kBand; n - 1 - kBand of them
        const int K1 = std::max(0, nb_ - 1 - kBand);
        L.npanel = (K1 + NBT - 1) / NBT;
        BandBlock Bb{};
        Bb.S = L.W1;
        Bb.H = L.H;
        Bb.lds = L.ldp;
        Bb.n = nb_;
        Bb.J = band_nsteps(nb_, 0);
        int jf = 0;
        while (nb_ - jf - kBand > 1) jf += kBand;
        Bb.jfin = jf;
        Bb.BND = take((size_t)nb_ * kLDB);
        Bb.V2 = take((size_t)band_nsweeps(nb_) * Bb.J * kBand);
        Bb.tau2 = take((size_t)band_nsweeps(nb_) * Bb.J);
        Bb.T2 = take((size_t)band_ngroups(nb_) * Bb.J * kGrp * kGrp);
        Bb.tau1 = L.tau;
        Bb.scr = L.W2;
        Bb.d = L.d;
        Bb.e = L.e;
        Bb.evecs = L.evecs;
        Bb.info = L.info;
        bblk.push_back(Bb);
        shift.push_back(kBand);
      } else {
        shift.push_back(1);
      }
      blk.push_back(L);
      maxn = std::max(maxn, nb_);
      maxpanel = std::max(maxpanel, L.npanel);
    }
    const int nb = (int)blk.size();
    if (off > c->ws_size) return fail(NRG_ERR_ARG, "internal: chunk workspace %zu > %zu", off, c->ws_size);
    // ---- 2-D tensor maps over each block's packed lower triangle (box 64 rows x 8 columns)
    std::vector<CUtensorMap> tmaps(nb);
    {
      auto encode = tensor_map_encoder();
      if (!encode) return fail(NRG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
      for (int bi = nts; bi < nb; bi++) {
        const LargeBlock& L = blk[bi];
        if (L.n <= mid_max_n) continue;  // reduced in the shared memory of one CTA, no bulk copies
        const cuuint64_t dims[2] = {(cuuint64_t)L.ldp, (cuuint64_t)L.n};
        const cuuint64_t strides[1] = {(cuuint64_t)L.ldp * sizeof(double)};
        const cuuint32_t box[2] = {(cuuint32_t)kSlabRows, 8u};
        const cuuint32_t estr[2] = {1u, 1u};
        const CUresult r = encode(&tmaps[bi], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, L.W1, dims, strides, box, estr,
                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return fail(NRG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for n=%d", (int)r, L.n);
      }
    }
    // ---- divide-and-conquer tree (leaves and merge levels by height)
    std::vector<DcLeaf> leaves;
    std::vector<std::vector<DcNode>> levels;
    std::function<int(int, int, int)> build = [&](int bi, int lo, int hi) -> int {
      if (hi - lo <= kLeaf) {
        leaves.push_back(DcLeaf{bi, lo, hi, 0});
        return 0;
      }
      const int mid = lo + (hi - lo) / 2;
      const int h = 1 + std::max(build(bi, lo, mid), build(bi, mid, hi));
      if ((int)levels.size() < h) levels.resize(h);
      DcNode nd{};
      nd.blk = bi;
      nd.a = lo;
      nd.m = mid;
      nd.b = hi;
      levels[h - 1].push_back(nd);
      return h;
    };
    for (int bi = 0; bi < nb; bi++) build(bi, 0, blk[bi].n);
    // ---- one staging image for the whole chunk
    std::vector<char> img;
    const size_t blk_off = push(img, blk);
    const size_t tmap_off = push(img, tmaps);
    const size_t leaf_off = push(img, leaves);
    std::vector<size_t> node_off(levels.size()), st_off(levels.size());
    std::vector<StagedGemm> lvl_gemm(levels.size());
    for (size_t h = 0; h < levels.size(); h++) {
      GemmPlan gp;
      for (auto& nd : levels[h]) {
        const LargeBlock& L = blk[nd.blk];
        const int N = nd.b - nd.a, nn = L.n;
        nd.gout = (int)gp.outs.size();
        // child-1 columns: C = Zt[a:a+K, a:m] = U[:, 0:k1+k2] * G[a:a+k1+k2, a:m]
        gp.add_out(L.H + (size_t)nd.a * nn + nd.a, nn, N, nd.m - nd.a, 0.0);
        gp.add_seg(L.evecs + (size_t)nd.a * nn + nd.a, nn, 0, L.W2 + (size_t)nd.a * nn + nd.a, nn, 0, N, 1.0);
        // child-2 columns: C = Zt[a:a+K, m:b] = U[:, k1:K] * G[a+k1:a+K, m:b] (pointers set on device)
        gp.add_out(L.H + (size_t)nd.a * nn + nd.m, nn, N, nd.b - nd.m, 0.0);
        gp.add_seg(L.evecs + (size_t)nd.a * nn + nd.a, nn, 0, L.W2 + (size_t)nd.a * nn + nd.m, nn, 0, N, 1.0);
      }
      node_off[h] = push(img, levels[h]);
      st_off[h] = push(img, std::vector<DcState>(levels[h].size()));
      lvl_gemm[h] = stage_gemm(img, gp);
    }
    // back-transform: Gram, T, VT, then per panel step two GEMMs
    std::vector<PanelRef> panels;
    GemmPlan gram, vt;
    std::vector<GemmPlan> bsteps(maxpanel * 2);
    for (int bi = 0; bi < nb; bi++) {
      const LargeBlock& L = blk[bi];
      const int nn = L.n;
      size_t vt_off = 0, gt_off = 0;
      // reflector k has its unit at row k + sh: k + 1 after the one-stage reduction, k + kBand
      // after the first stage of the two-stage one; nn - 1 - sh reflectors
      const int sh = shift[bi], nrefl = nn - 1 - sh;
      for (int p = 0; p < L.npanel; p++) {
        const int k0 = p * NBT, pnb = std::min(NBT, nrefl - k0), K = nn - k0 - sh;
        panels.push_back(PanelRef{bi, k0, pnb, 0, (long long)gt_off});
        double* Gp = L.GT + gt_off;                 // pnb x pnb
        double* Tp = Gp + (size_t)pnb * pnb;        // pnb x pnb
        gt_off += 2 * (size_t)pnb * pnb;
        const double* Vrows = L.W1 + (size_t)k0 * L.ldp + k0 + sh;  // pnb x K, row q = v_{k0+q}
        gram.add_out(Gp, pnb, pnb, pnb, 0.0);
        gram.add_seg(Vrows, L.ldp, 0, Vrows, L.ldp, 1, K, 1.0);
        double* VTp = L.H + vt_off;  // K x pnb (H is free after the final row permutation)
        vt_off += (size_t)K * pnb;
        if (vt_off > (size_t)nn * nn) return fail(NRG_ERR_ARG, "internal: VT factors exceed H for n=%d", nn);
        vt.add_out(VTp, pnb, K, pnb, 0.0);
        vt.add_seg(Vrows, L.ldp, 1, Tp, pnb, 0, pnb, 1.0);
        // step index counts from the last panel of each block
        const int stp = L.npanel - 1 - p;
        GemmPlan& g1 = bsteps[2 * stp];
        GemmPlan& g2 = bsteps[2 * stp + 1];
        double* Wb = L.W2;  // n x pnb
        g1.add_out(Wb, pnb, nn, pnb, 0.0);
        g1.add_seg(L.evecs + k0 + sh, nn, 0, Vrows, L.ldp, 1, K, 1.0);
        g2.add_out(L.evecs + k0 + sh, nn, nn, K, 1.0);
        g2.add_seg(Wb, pnb, 0, VTp, pnb, 1, pnb, -1.0);
      }
    }
    const size_t pan_off = push(img, panels);
    // two-stage blocks: per stage-1 panel j0 = p kBand, the blocks with more than one row below
    // the band (a prefix: sorted by order), six GEMMs of the trailing update in compact-WY form
    //   X = S22 V, Y = X T1, Z = V^T Y, U = T1^T Z, W = Y - V U / 2, S22 -= V W^T + W V^T
    const size_t bblk_off = push(img, bblk);
    int npan1 = 0;
    for (const BandBlock& Bb : bblk) npan1 = std::max(npan1, Bb.jfin / kBand);
    std::vector<int> pan_active(npan1, 0);
    std::vector<StagedGemm> s1_g((size_t)npan1 * 6);
    for (int p = 0; p < npan1; p++) {
      const int j0 = p * kBand;
      GemmPlan ga, gb, gc, gd, ge, gf;
      for (const BandBlock& Bb : bblk) {
        const int nn = Bb.n, m = nn - j0 - kBand;
        if (m <= 1) break;
        pan_active[p]++;
        const int kb = std::min(kBand, m - 1);
        double* S22 = Bb.S + (size_t)(j0 + kBand) * Bb.lds + j0 + kBand;
        const double* Vt = Bb.S + (size_t)j0 * Bb.lds + j0 + kBand;  // kb x m
        double* Y = Bb.scr + band_scr_y(nn);
        double* T1 = Bb.scr + band_scr_t(nn);
        double* U = Bb.scr + band_scr_u(nn);
        const int ns = band_split(m), chunk = (m + ns - 1) / ns;
        // X = S22 V and Z = V^T Y in parts along m (rows k0 .. k1 of V), summed as segments
        for (int q = 0; q < ns; q++) {
          const int k0 = q * chunk, k1 = std::min(m, k0 + chunk);
          if (k1 <= k0) break;
          double* Xq = Bb.scr + band_scr_x(nn, q);
          ga.add_out(Xq, kBand, m, kb, 0.0);
          ga.add_seg(S22 + k0, Bb.lds, 0, Vt + k0, Bb.lds, 1, k1 - k0, 1.0);
        }
        gb.add_out(Y, kBand, m, kb, 0.0);
        for (int q = 0; q < ns; q++) {
          if (q * chunk >= m) break;
          gb.add_seg(Bb.scr + band_scr_x(nn, q), kBand, 0, T1, kBand, 0, kb, 1.0);
        }
        for (int q = 0; q < ns; q++) {
          const int k0 = q * chunk, k1 = std::min(m, k0 + chunk);
          if (k1 <= k0) break;
          gc.add_out(Bb.scr + band_scr_z(nn, q), kBand, kb, kb, 0.0);
          gc.add_seg(Vt + k0, Bb.lds, 0, Y + (size_t)k0 * kBand, kBand, 0, k1 - k0, 1.0);
        }
        gd.add_out(U, kBand, kb, kb, 0.0);
        for (int q = 0; q < ns; q++) {
          if (q * chunk >= m) break;
          gd.add_seg(T1, kBand, 1, Bb.scr + band_scr_z(nn, q), kBand, 0, kb, 1.0);
        }
        ge.add_out(Y, kBand, m, kb, 1.0);
        ge.add_seg(Vt, Bb.lds, 1, U, kBand, 0, kb, -0.5);
        gf.add_out(S22, Bb.lds, m, m, 1.0);
        gf.add_seg(Vt, Bb.lds, 1, Y, kBand, 1, kb, -1.0);
        gf.add_seg(Y, kBand, 0, Vt, Bb.lds, 0, kb, -1.0);
      }
      s1_g[6 * p + 0] = stage_gemm(img, ga);
      s1_g[6 * p + 1] = stage_gemm(img, gb);
      s1_g[6 * p + 2] = stage_gemm(img, gc);
      s1_g[6 * p + 3] = stage_gemm(img, gd);
      s1_g[6 * p + 4] = stage_gemm(img, ge);
      s1_g[6 * p + 5] = stage_gemm(img, gf);
    }
    const StagedGemm gram_g = stage_gemm(img, gram), vt_g = stage_gemm(img, vt);
    std::vector<StagedGemm> bs_g(bsteps.size());
    for (size_t t = 0; t < bsteps.size(); t++) bs_g[t] = stage_gemm(img, bsteps[t]);
    rc = stage_desc(c, img, s);
    if (rc) return rc;
    char* dbase = static_cast<char*>(c->desc);
    const LargeBlock* dblk = reinterpret_cast<const LargeBlock*>(dbase + blk_off);
    const BandBlock* dbb = reinterpret_cast<const BandBlock*>(dbase + bblk_off);

    // ---- 1a. two-stage reduction of the largest blocks (when few): symmetric copy, stage-1
    //          panels and their GEMMs, bulge chasing, the T factors of its back-transform.
    //          With one-stage blocks beside them it runs on the context's fourth stream, so
    //          that the one-stage reductions fill the SMs its clusters leave idle.
    const bool fork3 = nts > 0 && nts < nb;
    cudaStream_t s3 = s;
    if (fork3) {
      if (!c->side3) {
        NRG_CK(cudaStreamCreateWithFlags(&c->side3, cudaStreamNonBlocking));
        NRG_CK(cudaEventCreateWithFlags(&c->fork3_ev, cudaEventDisableTiming));
        NRG_CK(cudaEventCreateWithFlags(&c->join3_ev, cudaEventDisableTiming));
      }
      NRG_CK(cudaEventRecord(c->fork3_ev, s));
      NRG_CK(cudaStreamWaitEvent(c->side3, c->fork3_ev, 0));
      s3 = c->side3;
    }
    if (nts > 0) {
      for (const BandBlock& Bb : bblk)
        NRG_CK(cudaMemsetAsync(Bb.BND, 0, sizeof(double) * (size_t)Bb.n * kLDB, s3));
      {
        PhaseScope ps(c, kPhBandReduce, s3);
        NRG_CK(band_sym_launch(dbb, nts, blk[0].n, s3));
      }
      for (int p = 0; p < npan1; p++) {
        {
          PhaseScope ps(c, kPhBandPanel, s3);
          NRG_CK(band_panel_launch(dbb, pan_active[p], p * kBand, bblk[0].n - p * kBand - kBand, s3));
        }
        for (int q = 0; q < 6; q++) {
          rc = launch_staged_gemm(c, s1_g[6 * p + q], s3, kPhBandReduce);
          if (rc) return rc;
        }
      }
      {
        PhaseScope ps(c, kPhBulgeChase, s3, 2);
        NRG_CK(band_chase_launch(dbb, nts, s3));
        NRG_CK(band_q2_tfactor_launch(dbb, nts, blk[0].n, s3));
      }
      if (fork3) NRG_CK(cudaEventRecord(c->join3_ev, s3));
    }

    // ---- 1. tridiagonalisation: blocks beyond cluster_max_n (sorted first) stream through
    //         TMA, blocks beyond mid_max_n are spread over the shared memory of a cluster,
    //         the rest are reduced in the shared memory of one CTA
    {
      int nsm = 148;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
      // the one-stage reductions: the blocks after the two-stage ones
      const LargeBlock* b1 = blk.data() + nts;
      const LargeBlock* d1 = dblk + nts;
      const int nb1 = nb - nts;
      int nbig = 0;
      while (nbig < nb1 && b1[nbig].n > cluster_max_n) nbig++;
      int nclu = nbig;
      while (nclu < nb1 && b1[nclu].n > mid_max_n) nclu++;
      // One cluster size for all cluster blocks (one launch): the smallest of 2, 4, 8 that
      // fits the largest of them, raised while the cluster CTAs still fit the SMs once. The
      // clusters serve latency: when they would not all fit the SMs at once (a batch of many
      // blocks), the blocks go to the bulk-copy kernel, whose two CTAs per SM give more
      // throughput.
      int C = 0;
      if (nclu > nbig) {
        for (int q = 2; q <= 8 && !C; q *= 2)
          if (sizeof(double) * cl_smem_doubles(b1[nbig].n, q) <= 232448) C = q;
        if (C == 0) return fail(NRG_ERR_ARG, "internal: no cluster size for n=%d", b1[nbig].n);
        if (C * (nclu - nbig) > nsm) {
          nbig = nclu;  // throughput regime
          C = 0;
        } else {
          while (C < 8 && 2 * C * (nclu - nbig) <= nsm) C *= 2;
        }
      }
      const bool fork = nb1 > nclu && (nbig > 0 || nclu > nbig);
      if (fork && !c->side2) {
        NRG_CK(cudaStreamCreateWithFlags(&c->side2, cudaStreamNonBlocking));
        NRG_CK(cudaEventCreateWithFlags(&c->fork2_ev, cudaEventDisableTiming));
        NRG_CK(cudaEventCreateWithFlags(&c->join2_ev, cudaEventDisableTiming));
      }
      PhaseScope ps(c, kPhTridiag, s, (nbig ? 2 : 0) + (nclu > nbig ? 1 : 0) + (nb1 > nclu ? 1 : 0));
      if (nb1 > nclu) {  // one CTA per block, on the third stream when other launches run beside it
        cudaStream_t ss = s;
        if (fork) {
          NRG_CK(cudaEventRecord(c->fork2_ev, s));
          NRG_CK(cudaStreamWaitEvent(c->side2, c->fork2_ev, 0));
          ss = c->side2;
        }
        const int mn = b1[nclu].n;
        const size_t smem = sizeof(double) * ((size_t)mn * (mn + 1) / 2 + 2 * (size_t)mn + 64);
        NRG_CK(cudaFuncSetAttribute(tridiag_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        tridiag_smem_kernel<<<nb1 - nclu, kMidThreads, smem, ss>>>(d1 + nclu);
        NRG_CK(cudaGetLastError());
        if (fork) NRG_CK(cudaEventRecord(c->join2_ev, ss));
      }
      if (nclu > nbig) {
        const long long ld0 = cl_smem_doubles(b1[nbig].n, C);  // the largest block sets the layout
        const int lmax = (int)(ld0 - (4LL * b1[nbig].n + 64));
        const size_t smem = sizeof(double) * (size_t)ld0;
        NRG_CK(cudaFuncSetAttribute(tridiag_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)((nclu - nbig) * C));
        cfg.blockDim = dim3(kClThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)C;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        NRG_CK(cudaLaunchKernelEx(&cfg, tridiag_cluster_kernel, d1 + nbig, lmax));
      }
      if (nbig) {
        auto tri_bytes = [&](int st) {
          return 1024 + sizeof(double) * ((size_t)kTriWarps * st * kSlabD + 2 * (size_t)b1[0].n +
                                          (size_t)kTriWarps * 2 * NB + 2 * NB + 64);
        };
        const CUtensorMap* tm = reinterpret_cast<const CUtensorMap*>(dbase + tmap_off) + nts;
        pack_lower_kernel<<<dim3((b1[0].n + 7) / 8, nbig), 256, 0, s>>>(d1);
        NRG_CK(cudaGetLastError());
        // Few large blocks: one cluster of kTclC CTAs per block, when the clusters fill at most
        // about two waves of the SMs and the device can hold one such cluster at a time.
        bool tcl = false;
        // reduction_ctas_per_sm (nrg_tuning) sets how many CTAs of the streaming kernel share an
        // SM: one, when each requests at least half of an SM's shared memory; two, with four
        // slabs in flight per warp; three (the default), with two slabs per warp and at most 168
        // registers per thread. More CTAs per SM keep the SM's HBM stream going while a CTA is
        // in the serial part of a column (norm, reflector, block sums); where the blocks' vectors
        // leave no room for that many, the next smaller count is used. Several per SM once gave
        // wrong reductions through a race on alpha = v[k+1] in the reflector step (alpha was read
        // after a barrier that a thread overwriting it could pass); alpha is now read before that
        // barrier, and batches with more of these CTAs than SMs pass every check on B200. The
        // cluster kernel's ring gets 8, 6 or 4 slabs per warp, the most that fit.
        int smsm = 0, optin = 0;
        cudaDeviceGetAttribute(&smsm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
        // The cluster kernel serves few blocks (latency): its CTAs keep an SM each, whatever
        // reduction_ctas_per_sm says for the streaming kernel of the throughput regime.
        auto tcl_bytes = [&](int st) {
          return std::max(1024 + sizeof(double) * ((size_t)kTriWarps * st * kSlabD + 2 * (size_t)b1[0].n +
                                                   (size_t)kTriWarps * 2 * NB + 4 * NB + 66),
                          (size_t)smsm / 2 + 1024);
        };
        int stages = 8;
        while (stages > 4 && tcl_bytes(stages) + 256 > (size_t)optin) stages -= 2;
        const size_t smem_tcl = tcl_bytes(stages);
        const void* tcl_fn = stages == 8 ? (const void*)tridiag_tcl_kernel<8>
                             : stages == 6 ? (const void*)tridiag_tcl_kernel<6> : (const void*)tridiag_tcl_kernel<4>;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        if ((long long)nbig * kTclC <= 2LL * nsm && smem_tcl + 256 <= (size_t)optin) {
          NRG_CK(cudaFuncSetAttribute(tcl_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tcl));
          NRG_CK(cudaFuncSetAttribute(tcl_fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
          cfg.blockDim = dim3(kTriThreads);
          cfg.dynamicSmemBytes = smem_tcl;
          cfg.stream = s;
          at[0].id = cudaLaunchAttributeClusterDimension;
          at[0].val.clusterDim.y = 1;
          at[0].val.clusterDim.z = 1;
          cfg.attrs = at;
          cfg.numAttrs = 1;
          // 16 CTAs per block when the blocks are few enough for all their clusters to be active
          // at once, else 8
          for (int C : {2 * kTclC, kTclC}) {
            if (C > kTclC && (long long)nbig * C > nsm) continue;
            cfg.gridDim = dim3((unsigned)(nbig * C));
            at[0].val.clusterDim.x = (unsigned)C;
            int ncl = 0;
            if (cudaOccupancyMaxActiveClusters(&ncl, tcl_fn, &cfg) != cudaSuccess) {
              cudaGetLastError();
              ncl = 0;
            }
            if (C > kTclC ? ncl >= nbig : ncl > 0) {
              tcl = true;
              break;
            }
          }
        }
        if (tcl) {
          const LargeBlock* db = d1;
          void* kargs[] = {(void*)&db, (void*)&tm};
          NRG_CK(cudaLaunchKernelExC(&cfg, tcl_fn, kargs));
        } else {
          // one, two or three CTAs per SM as above (1 KB of shared memory is reserved per CTA);
          // reduction_ctas_per_sm is the most, used when the batch fills at least three waves of
          // that many CTAs per SM. A batch of fewer large blocks is bound by its largest ones,
          // which finish sooner with an SM's bandwidth shared by fewer CTAs (measured on B200:
          // 1500 blocks of order 8-2048, about 330 of them streamed, take 873 ms with one CTA
          // per SM, 909 with two, 1015 with three; the benchmark's 10,000 blocks run 6.5% faster
          // with three than with two).
          int per_sm = c->tune.reduction_ctas_per_sm;
          while (per_sm > 1 && (long long)nbig < 3LL * per_sm * nsm) per_sm--;
          if (per_sm == 3 && 3 * (tri_bytes(2) + 1024) > (size_t)smsm) per_sm = 2;
          if (per_sm == 2 && 2 * (tri_bytes(4) + 1024) > (size_t)smsm) per_sm = 1;
          if (per_sm == 3) {
            const size_t smem3 = tri_bytes(2);
            NRG_CK(cudaFuncSetAttribute(tridiag_kernel<2, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem3));
            tridiag_kernel<2, 3><<<nbig, kTriThreads, smem3, s>>>(d1, tm);
          } else {
            const size_t smem1 = std::max(tri_bytes(4), (per_sm == 1 ? (size_t)smsm / 2 + 1024 : (size_t)0));
            NRG_CK(cudaFuncSetAttribute(tridiag_kernel<4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem1));
            tridiag_kernel<4, 2><<<nbig, kTriThreads, smem1, s>>>(d1, tm);
          }
          NRG_CK(cudaGetLastError());
        }
      }
      if (fork) NRG_CK(cudaStreamWaitEvent(s, c->join2_ev, 0));
    }
    if (fork3) NRG_CK(cudaStreamWaitEvent(s, c->join3_ev, 0));  // the two-stage blocks are tridiagonal
    // ---- 2. divide and conquer
    {
      PhaseScope ps(c, kPhDcLeaf, s);
      dc_leaf_kernel<<<(int)leaves.size(), 128, 0, s>>>(dblk, reinterpret_cast<const DcLeaf*>(dbase + leaf_off));
      NRG_CK(cudaGetLastError());
    }
    for (size_t h = 0; h < levels.size(); h++) {
      int maxN = 0;
      for (auto& nd : levels[h]) maxN = std::max(maxN, nd.b - nd.a);
      const int nn = (int)levels[h].size();
      const DcNode* dn = reinterpret_cast<const DcNode*>(dbase + node_off[h]);
      DcState* dst = reinterpret_cast<DcState*>(dbase + st_off[h]);
      GemmOut* go = reinterpret_cast<GemmOut*>(dbase + lvl_gemm[h].outs_off);
      GemmSeg* gs = reinterpret_cast<GemmSeg*>(dbase + lvl_gemm[h].segs_off);
      // shared memory for the largest node that fits it; larger nodes use global scratch
      size_t ps = 16;
      for (auto& nd : levels[h]) {
        const size_t t = prep_layout(nd.b - nd.a).total;
        if (t <= kPrepSmemMax) ps = std::max(ps, t);
      }
      NRG_CK(cudaFuncSetAttribute(dc_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ps));
      {
        PhaseScope sc(c, kPhDcPrep, s);
        dc_prep_kernel<<<nn, 512, ps, s>>>(dblk, dn, dst, go, gs, ps);
        NRG_CK(cudaGetLastError());
      }
      // one warp per root (8 per CTA), at most 64 CTAs per node
      const int ysplit = std::max(1, std::min(64, (maxN + 7) / 8));
      {
        PhaseScope sc(c, kPhDcSecular, s);
        dc_secular_kernel<<<dim3(nn, ysplit), 256, 0, s>>>(dblk, dn, dst);
        NRG_CK(cudaGetLastError());
      }
      {
        PhaseScope sc(c, kPhDcVectors, s, 2);
        dc_zhat_kernel<<<dim3(nn, std::max(1, (maxN + 255) / 256)), 256, 0, s>>>(dblk, dn, dst);
        NRG_CK(cudaGetLastError());
        dc_vectors_kernel<<<dim3(nn, ysplit), 256, 0, s>>>(dblk, dn, dst);
        NRG_CK(cudaGetLastError());
      }
      rc = launch_staged_gemm(c, lvl_gemm[h], s, kPhDcGemm);
      if (rc) return rc;
    }
    // ---- 3. order
    {
      int P = 1;
      while (P < maxn) P <<= 1;
      const size_t ss = (sizeof(double) + sizeof(int)) * (size_t)P;
      NRG_CK(cudaFuncSetAttribute(sort_final_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
      PhaseScope sc(c, kPhSort, s, 2);
      sort_final_kernel<<<nb, 1024, ss, s>>>(dblk);
      NRG_CK(cudaGetLastError());
      permute_rows_kernel<<<dim3((maxn + 7) / 8, nb), 256, 0, s>>>(dblk);
      NRG_CK(cudaGetLastError());
    }
    // ---- 3a. two-stage blocks: the bulge-chasing reflectors applied to the eigenvector rows
    if (nts > 0) {
      PhaseScope sc(c, kPhBtBand, s);
      NRG_CK(band_q2_apply_launch(dbb, nts, blk[0].n, s));
    }
    // ---- 4. back-transform
    rc = launch_staged_gemm(c, gram_g, s, kPhBtGemm);
    if (rc) return rc;
    if (!panels.empty()) {
      PhaseScope sc(c, kPhBtTfactor, s);
      const size_t ts = sizeof(double) * ((size_t)NBT * (NBT + 1) + NBT);
      NRG_CK(cudaFuncSetAttribute(tfactor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ts));
      tfactor_kernel<<<(int)panels.size(), NBT, ts, s>>>(dblk, reinterpret_cast<const PanelRef*>(dbase + pan_off));
      NRG_CK(cudaGetLastError());
    }
    rc = launch_staged_gemm(c, vt_g, s, kPhBtGemm);
    if (rc) return rc;
    for (size_t t = 0; t < bs_g.size(); t++) {
      rc = launch_staged_gemm(c, bs_g[t], s, kPhBtGemm);
      if (rc) return rc;
    }
    pos = end;
    if (pos < ord.size()) NRG_CK(cudaStreamSynchronize(s));  // the next chunk reuses the workspace
  }
  return NRG_OK;
}

}  // namespace nrg
