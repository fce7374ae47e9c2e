// kernels.h -- internal host-side launch interface between the C-ABI layer and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrg_b200.h"

namespace nrg {

// ---------------------------------------------------------------- batched FP64 GEMM
// One K-segment of an output: alpha * op(A) * op(B), op(A) is M x K, op(B) is K x N.
// transA: A is stored K x M row-major (op(A) = A^T); transB: B is stored N x K (op(B) = B^T).
struct GemmSeg {
  const double* A;
  const double* B;
  int64_t lda, ldb;
  int K, transA, transB, pad_;
  double alpha;
};

// T = diag(d) op(B) for one term (rows x cols, row-major, ld = cols); off is the term's first
// element in the batch's flattened element range.
struct RowScale {
  double* T;
  const double* d;
  const double* B;
  int64_t ldb, off;
  int rows, cols, transB, pad_;
};
cudaError_t row_scale_launch(const RowScale* d_terms, int nterm, int64_t total, cudaStream_t stream);

// One output C (M x N, row-major, ldc): C = beta*C + sum over its segments. Tiles of
// 64 x 64 are numbered from tile0 in row-major tile order.
struct GemmOut {
  double* C;
  int64_t ldc;
  int M, N;
  int seg0, nseg;
  int tile0, pad_;
  double beta;
};

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16, kGemmThreads = 128;

// Launch over nout outputs whose descriptors already live in device memory.
cudaError_t gemm_batch_launch(const GemmOut* d_outs, const GemmSeg* d_segs, int nout, int ntiles,
                              cudaStream_t stream);
// One output C = beta*C + alpha op(A) op(B) with descriptors passed as kernel parameters.
cudaError_t gemm_one_launch(const GemmOut& o, const GemmSeg& g, cudaStream_t stream);

// ---------------------------------------------------------------- eigensolver
// Per-block descriptor of the batched symmetric eigensolver. H is n x n row-major with the
// upper triangle set (it is overwritten); evals n doubles; evecs n x n row-major, row r =
// eigenvector r. W1/W2 are n x n workspaces (large path only); d, e, tau are n-vectors.
struct EigBlock {
  double* H;
  double* evals;
  double* evecs;
  double* W1;
  double* W2;
  double* d;
  double* e;
  double* tau;
  int* iwork;     // 4n ints (large path)
  int* info;      // per-block status word (0 ok, >0 not converged, <0 invalid)
  int n, pad_;
};

constexpr int kSmallMaxN = 64;   // default: blocks up to this size are solved entirely in shared memory
constexpr int kSmallMaxNLimit = 96;  // the most the one-CTA solver's shared memory holds
constexpr int kMidMaxN = 224;        // default: one-CTA shared-memory reduction up to this order
constexpr int kMidMaxNLimit = 236;   // the packed triangle of the most the 227 KB of one CTA holds
constexpr int kClusterMaxN = 600;    // default: cluster (distributed shared memory) reduction up to here
constexpr int kClusterMaxNLimit = 640;  // the most an 8-CTA cluster's shared memory holds

cudaError_t eig_small_launch(const EigBlock* d_blocks, int nblk, int maxn, cudaStream_t stream);

// ---------------------------------------------------------------- Hamiltonian assembly
// One block of nrg_hamiltonian_batch: its matrix, order, first tile and its pieces
// [p0, p1) in the sorted piece array.
struct HBlock {
  double* H;
  int n, tile0, p0, p1;
};
int hamiltonian_tiles(int n);
cudaError_t hamiltonian_launch(const HBlock* d_blocks, int nblk, int ntiles, const nrg_hpiece* d_pieces,
                               cudaStream_t stream);

// ---------------------------------------------------------------- spectrum broadening
cudaError_t broaden_launch(int nspike, const double* e, const double* w, int nmesh, const double* E, double alpha,
                           double omega0, double* out, cudaStream_t stream);

}  // namespace nrg
