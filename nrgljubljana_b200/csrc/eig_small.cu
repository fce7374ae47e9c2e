// eig_small.cu -- one CTA per block, whole eigenproblem in shared memory (n <= kSmallMaxN).
//
// Replaces LAPACK dsyev as called by diagonalise_dsyev (c++/diag.hpp:62-82 of the
// reference) for the small symmetry blocks of an NRG step: the row-major input with its
// upper triangle set is symmetrised into shared memory, reduced to tridiagonal form by
// Householder reflections, the orthogonal factor is formed explicitly, and the implicit
// QL iteration accumulates its rotations into it. Eigenvalues are written ascending and
// eigenvectors as rows (the layout of copy_vec, c++/diag.hpp:41-48).
#include "eig_small.cuh"
#include "kernels.h"

namespace nrg {
namespace {

constexpr int kThreads = 128;

__host__ __device__ inline int small_ld(int n) { return (n & 1) ? n : n + 1; }  // odd stride: no bank conflicts

__host__ __device__ inline size_t small_smem_bytes(int n) {
  const int ld = small_ld(n);
  return sizeof(double) * (2 * (size_t)n * ld + 10 * (size_t)n + 32) + sizeof(int) * ((size_t)n + 8);
}

__global__ void __launch_bounds__(kThreads) eig_small_kernel(const EigBlock* __restrict__ blocks) {
  extern __shared__ __align__(16) double sm[];
  const EigBlock b = blocks[blockIdx.x];
  const int n = b.n, ld = small_ld(n), tid = threadIdx.x, nt = blockDim.x;
  double* A = sm;
  double* Z = A + (size_t)n * ld;
  double* d = Z + (size_t)n * ld;
  double* e = d + n;
  double* taus = e + n;
  double* vw = taus + n;  // 2n
  double* C = vw + 2 * n;  // 2n: two buffers of QL rotations
  double* S = C + 2 * n;   // 2n
  double* scr = S + 2 * n;  // n
  double* red = scr + n;  // 32
  int* ctl = reinterpret_cast<int*>(red + 32);  // 8
  int* perm = ctl + 8;                          // n

  // Load the upper triangle and symmetrise; flag non-finite input.
  int bad = 0;
  for (int idx = tid; idx < n * n; idx += nt) {
    const int i = idx / n, j = idx - i * n;
    if (j >= i) {
      const double h = b.H[idx];
      if (!isfinite(h)) bad = 1;
      A[i * ld + j] = h;
      A[j * ld + i] = h;
    }
  }
  const int anybad = __syncthreads_or(bad);

  smem_tridiagonalise(A, ld, n, d, e, taus, vw, red);
  smem_form_q(A, ld, n, taus, Z, scr);
  const int st = smem_ql(d, e, n, Z, ld, n, C, S, ctl);

  if (tid == 0) {
    serial_sort_perm(d, n, perm);
    *b.info = anybad ? -2 : st;
  }
  __syncthreads();
  for (int r = tid; r < n; r += nt) b.evals[r] = d[perm[r]];
  for (int idx = tid; idx < n * n; idx += nt) {
    const int r = idx / n, j = idx - r * n;
    b.evecs[idx] = Z[j * ld + perm[r]];
  }
}

}  // namespace

cudaError_t eig_small_launch(const EigBlock* d_blocks, int nblk, int maxn, cudaStream_t stream) {
  if (nblk <= 0) return cudaSuccess;
  const size_t smem = small_smem_bytes(maxn);
  cudaError_t err = cudaFuncSetAttribute(eig_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  eig_small_kernel<<<nblk, kThreads, smem, stream>>>(d_blocks);
  return cudaGetLastError();
}

}  // namespace nrg
