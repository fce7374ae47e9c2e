// assemble.cu -- batched assembly of the block Hamiltonians of one NRG step.
//
// Device counterpart of hamiltonian() (c++/core.hpp:72-88): every block H_I is cleared and
// the pieces that make_matrix() (c++/symmetry/sym-QS-impl.hpp:111-155) would add are
// accumulated in their given order -- the diagonal of the ancestor energies scaled by
// sqrt(Lambda) (c++/core.hpp:79-82), the zeta shifts of diag_function_impl
// (c++/matrix.hpp:67-78), the xi-scaled <||f||> blocks of offdiag_function_impl
// (c++/matrix.hpp:32-58) and the diagonal shifts of diag_offdiag_function
// (c++/matrix.hpp:97-111). Every product and sum is rounded separately (no FMA
// contraction) so that the matrix is bit-identical to the one the reference builds.
//
// HBM-bound: one pass of stores over n^2 doubles per block plus one read of each piece.
// A CTA owns a 32 x 128 tile of one block (rows of 1 KB, coalesced stores); it first
// gathers the pieces of its block that intersect the tile into shared memory, in order.
#include "common.cuh"
#include "kernels.h"

namespace nrg {
namespace {

constexpr int kTR = 32, kTC = 128, kThreads = 256;
constexpr int kMaxTilePieces = 128;

struct SPiece {
  const double* src;
  int64_t ld;
  double factor, shift;
  int r0, c0, rows, cols, kind, trans;
};

NRG_DEV bool intersects(const nrg_hpiece& p, int i0, int j0) {
  if (p.kind == NRG_HP_DIAG) {
    // diagonal run (r0 + k, c0 + k), k < rows, against rows [i0, i0+kTR), cols [j0, j0+kTC)
    const int klo = max(max(i0 - p.r0, j0 - p.c0), 0);
    const int khi = min(min(i0 + kTR - p.r0, j0 + kTC - p.c0), p.rows);
    return klo < khi;
  }
  return p.r0 < i0 + kTR && p.r0 + p.rows > i0 && p.c0 < j0 + kTC && p.c0 + p.cols > j0;
}

NRG_DEV double piece_value(const SPiece& p, int i, int j, double v) {
  const int a = i - p.r0, b = j - p.c0;
  if (p.kind == NRG_HP_DIAG) {
    if (a == b && a >= 0 && a < p.rows) {
      const double t = p.src ? __dmul_rn(p.factor, p.src[a]) : 0.0;
      v = __dadd_rn(v, __dadd_rn(t, p.shift));
    }
  } else if (a >= 0 && a < p.rows && b >= 0 && b < p.cols) {
    const double s = p.trans ? p.src[(int64_t)b * p.ld + a] : p.src[(int64_t)a * p.ld + b];
    v = __dadd_rn(v, __dmul_rn(p.factor, s));
  }
  return v;
}

NRG_DEV SPiece to_spiece(const nrg_hpiece& q) {
  SPiece p;
  p.src = q.src;
  p.ld = q.ld;
  p.factor = q.factor;
  p.shift = q.shift;
  p.r0 = q.r0;
  p.c0 = q.c0;
  p.rows = q.rows;
  p.cols = q.cols;
  p.kind = q.kind;
  p.trans = q.trans;
  return p;
}

__global__ void __launch_bounds__(kThreads) hamiltonian_kernel(const HBlock* __restrict__ blocks, int nblk,
                                                               const nrg_hpiece* __restrict__ pieces) {
  __shared__ SPiece list[kMaxTilePieces];
  __shared__ int wcount[kThreads / 32];
  __shared__ int s_cnt;
  const int t = blockIdx.x;
  int lo = 0, hi = nblk - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (blocks[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const HBlock hb = blocks[lo];
  const int lt = t - hb.tile0;
  const int tiles_c = (hb.n + kTC - 1) / kTC;
  const int i0 = (lt / tiles_c) * kTR, j0 = (lt % tiles_c) * kTC;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // Ordered compaction of the pieces that touch this tile.
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  bool overflow = false;
  for (int base = hb.p0; base < hb.p1; base += kThreads) {
    const int p = base + tid;
    const bool hit = p < hb.p1 && intersects(pieces[p], i0, j0);
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) wcount[warp] = __popc(m);
    __syncthreads();
    int off = s_cnt, total = 0;
    for (int w = 0; w < kThreads / 32; w++) {
      if (w < warp) off += wcount[w];
      total += wcount[w];
    }
    off += __popc(m & ((1u << lane) - 1u));
    if (hit && off < kMaxTilePieces) list[off] = to_spiece(pieces[p]);
    __syncthreads();
    if (tid == 0) s_cnt += total;
    __syncthreads();
  }
  const int cnt = s_cnt;
  overflow = cnt > kMaxTilePieces;

  const int j = j0 + (tid & (kTC - 1));
  for (int r = tid / kTC; r < kTR; r += kThreads / kTC) {
    const int i = i0 + r;
    if (i >= hb.n || j >= hb.n) continue;
    double v = 0.0;
    if (!overflow) {
      for (int k = 0; k < cnt; k++) v = piece_value(list[k], i, j, v);
    } else {
      // more pieces than the tile list holds: walk the block's whole list in order
      for (int p = hb.p0; p < hb.p1; p++) v = piece_value(to_spiece(pieces[p]), i, j, v);
    }
    hb.H[(int64_t)i * hb.n + j] = v;
  }
}

}  // namespace

int hamiltonian_tiles(int n) { return ((n + kTR - 1) / kTR) * ((n + kTC - 1) / kTC); }

cudaError_t hamiltonian_launch(const HBlock* d_blocks, int nblk, int ntiles, const nrg_hpiece* d_pieces,
                               cudaStream_t stream) {
  if (nblk <= 0 || ntiles <= 0) return cudaSuccess;
  hamiltonian_kernel<<<ntiles, kThreads, 0, stream>>>(d_blocks, nblk, d_pieces);
  return cudaGetLastError();
}

}  // namespace nrg
