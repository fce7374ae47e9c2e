// common.cuh -- shared device helpers for the NRG step core kernels (sm_100a, FP64).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define NRG_DEV __device__ __forceinline__

namespace nrg {

constexpr double kEps = 1.1102230246251565e-16;   // 2^-53, unit round-off of IEEE double
constexpr double kSafeMin = 2.2250738585072014e-308;

NRG_DEV double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

NRG_DEV double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum; `red` must hold one double per warp. Every thread gets the result.
NRG_DEV double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; w++) t += red[w];
  __syncthreads();
  return t;
}

// Block-wide sum with one barrier. `red` holds 64 doubles; `phase` is a per-thread counter
// that every thread of the block passes through the same sequence of calls, so consecutive
// calls use alternate halves of `red` and never overwrite values a slower thread may still
// be reading from the previous call.
NRG_DEV double block_sum_1b(double v, double* red, int& phase) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  double* buf = red + 32 * (phase & 1);
  phase++;
  if (lane == 0) buf[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; w++) t += buf[w];
  return t;
}

NRG_DEV double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; w++) t = fmax(t, red[w]);
  __syncthreads();
  return t;
}

// FP64 tensor-core MMA: D(8x8) += A(8x4) * B(4x8). Fragment layout (per lane l):
// a = A[l/4][l%4], b = B[l%4][l/4], d = {D[l/4][2*(l%4)], D[l/4][2*(l%4)+1]}.
NRG_DEV void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// FP64 tensor-core MMA: D(16x8) += A(16x16) * B(16x8). Fragment layout (per lane l,
// g = l/4, t = l%4): a[i] = A[g + 8*(i%2)][t + 4*(i/2)] (i < 8), b[i] = B[t + 4*i][g]
// (i < 4), d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}.
NRG_DEV void dmma16816(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}

}  // namespace nrg
