// band.h -- internal: the two-stage reduction of the largest symmetric blocks (dense ->
// band -> tridiagonal) and the back-transform of its second stage.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nrg {

constexpr int kBand = 32;              // bandwidth after stage 1 = reflector length of stage 2
constexpr int kGrp = 32;               // bulge-chasing sweeps per compact-WY group of the back-transform
constexpr int kLDB = 2 * kBand + 1;    // band storage per column: distances 0 .. 2 kBand below the diagonal
constexpr int kChaseWarps = 16;        // warps (sweeps in flight) per CTA of the bulge chasing
constexpr int kChaseCTAs = 4;          // CTAs (a cluster) per block in the bulge chasing

// Steps (reflectors) of bulge-chasing sweep i of an order-n band matrix: step j acts on rows
// i+1+j*kBand .. +kBand-1 (clipped at n) and exists while it has at least two rows.
__host__ __device__ inline int band_nsteps(int n, int i) { return i <= n - 3 ? (n - 3 - i) / kBand + 1 : 0; }
__host__ __device__ inline int band_nsweeps(int n) { return n > 2 ? n - 2 : 0; }
__host__ __device__ inline int band_ngroups(int n) { return (band_nsweeps(n) + kGrp - 1) / kGrp; }

// One block of the two-stage path.
struct BandBlock {
  double* S;          // n x lds: the full symmetric matrix during stage 1; row k then holds
                      // stage-1 reflector k in back-transform form (zeros, 1 at k+kBand, v)
  const double* H;    // the input (row-major, upper triangle)
  double* BND;        // n x kLDB: lower band, BND[c*kLDB + t] = A(c+t, c)
  double* V2;         // stage-2 reflectors: sweep i, step j at (i*J + j)*kBand (kBand entries)
  double* tau2;       // (i*J + j)
  double* T2;         // per group (g*J + j): kGrp x kGrp T factor of its reflectors
  double* tau1;       // stage-1 tau, indexed by reflector (column) k
  double* scr;        // stage-1 GEMM scratch (X, Y, T1, Z, U)
  double* d;          // tridiagonal result
  double* e;
  double* evecs;      // eigenvector rows (the stage-2 back-transform works on them)
  int* info;
  int n, lds, J, jfin;  // J = band_nsteps(n, 0); jfin: first column of the final diagonal block
};

// Stage-1 GEMMs whose inner dimension is the m rows below the band (X = S22 V and Z = V^T Y,
// both only kBand wide) are split along it into band_split(m) parts of about kSplitK, summed
// by the next GEMM as segments, so that they spread over the SMs.
constexpr int kSplitK = 256;
constexpr int kSplitMax = 32;
__host__ __device__ inline int band_split(int m) {
  const int s = (m + kSplitK - 1) / kSplitK;
  return s < 1 ? 1 : (s > kSplitMax ? kSplitMax : s);
}
// Stage-1 scratch layout inside BandBlock::scr (doubles; the block's n x n W2 buffer): Y
// (n x kBand), T1 and U (kBand x kBand each), the parts of Z (s0 x kBand x kBand) and of X
// (s0 x n x kBand), s0 = band_split(n - kBand) the most parts of any panel of the block.
__host__ __device__ inline size_t band_scr_y(int) { return 0; }
__host__ __device__ inline size_t band_scr_t(int n) { return (size_t)n * kBand; }
__host__ __device__ inline size_t band_scr_u(int n) { return (size_t)n * kBand + kBand * kBand; }
__host__ __device__ inline size_t band_scr_z(int n, int p) {
  return (size_t)n * kBand + (2 + (size_t)p) * kBand * kBand;
}
__host__ __device__ inline size_t band_scr_x(int n, int p) {
  return (size_t)n * kBand + (2 + (size_t)band_split(n - kBand)) * kBand * kBand + (size_t)p * n * kBand;
}
__host__ __device__ inline size_t band_scr_doubles(int n) { return band_scr_x(n, band_split(n - kBand)); }

// Device doubles of the stage-2 arrays of one block: band, reflectors, taus, T factors.
inline size_t band_extra_doubles(int n) {
  const size_t J = (size_t)band_nsteps(n, 0), S = (size_t)band_nsweeps(n), G = (size_t)band_ngroups(n);
  return (size_t)n * kLDB + S * J * kBand + S * J + G * J * kGrp * kGrp + 4 * 64;
}

cudaError_t band_sym_launch(const BandBlock* d_blocks, int nblk, int maxn, cudaStream_t s);
cudaError_t band_panel_launch(const BandBlock* d_blocks, int nactive, int j0, int mmax, cudaStream_t s);
cudaError_t band_chase_launch(const BandBlock* d_blocks, int nblk, cudaStream_t s);
cudaError_t band_q2_tfactor_launch(const BandBlock* d_blocks, int nblk, int maxn, cudaStream_t s);
cudaError_t band_q2_apply_launch(const BandBlock* d_blocks, int nblk, int maxn, cudaStream_t s);

}  // namespace nrg
