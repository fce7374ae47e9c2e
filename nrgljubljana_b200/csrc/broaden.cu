// broaden.cu -- log-Gaussian broadening of a binned spectrum onto an energy mesh.
//
// Device counterpart of SpectrumRealFreq::continuous() (c++/spectrum.hpp:168-196) with the
// kernel BR_NEW (c++/spectral.hpp:42-70): out[k] = sum_s w[s] BR_NEW(E[k], e[s]). One CTA
// per mesh point; each thread sums a fixed stride of the peaks and the CTA reduces in a
// fixed tree, so the result does not depend on scheduling.
#include "common.cuh"
#include "kernels.h"

namespace nrg {
namespace {

constexpr int kBrThreads = 256;
constexpr double kSqrtPi = 1.7724538509055160273;

NRG_DEV double br_new(double e, double ept, double alpha, double omega0) {
  double part_l = 0.0;
  if (!((e < 0.0 && ept > 0.0) || (e > 0.0 && ept < 0.0) || ept == 0.0)) {
    const double gamma = alpha / 4.0;
    const double t = log(e / ept) / alpha - gamma;
    part_l = exp(-t * t) / (alpha * fabs(e) * kSqrtPi);
  }
  if (fabs(e) > omega0) return part_l;
  const double u = log(fabs(e) / omega0) / alpha;
  const double br_h = exp(-u * u);
  const double g = (e - ept) / omega0;
  return part_l * br_h + exp(-g * g) / (omega0 * kSqrtPi) * (1.0 - br_h);
}

__global__ void __launch_bounds__(kBrThreads) broaden_kernel(int nspike, const double* __restrict__ e,
                                                             const double* __restrict__ w, const double* __restrict__ E,
                                                             double alpha, double omega0, double* __restrict__ out) {
  __shared__ double red[32];
  const double x = E[blockIdx.x];
  double s = 0.0;
  for (int i = threadIdx.x; i < nspike; i += blockDim.x) s += w[i] * br_new(x, e[i], alpha, omega0);
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

}  // namespace

cudaError_t broaden_launch(int nspike, const double* e, const double* w, int nmesh, const double* E, double alpha,
                           double omega0, double* out, cudaStream_t stream) {
  if (nmesh <= 0) return cudaSuccess;
  broaden_kernel<<<nmesh, kBrThreads, 0, stream>>>(nspike, e, w, E, alpha, omega0, out);
  return cudaGetLastError();
}

}  // namespace nrg
