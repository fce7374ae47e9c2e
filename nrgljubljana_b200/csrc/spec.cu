// spec.cu -- fused spectral-weight + log-grid binning kernel, and the Matsubara sums.
//
// Replaces the per-term loops of Algo_DMNRG::calc (c++/algo_DMNRG.hpp:29-52) and
// Algo_FDMgt/Algo_FDMls::calc (c++/algo_FDM.hpp:84-114, 30-60) together with
// ChainBinning::add (c++/spectrum.hpp:19-28) and Bins::add/add_std (c++/bins.hpp:103-132).
// The O(k^3) inner sums of the DM-NRG loop and the prod_fit products of FDM are computed
// beforehand as GEMMs (X, Y); this kernel only forms the weights and scatters them.
//
// Every CTA keeps a private copy of both sign halves of the histogram in shared memory
// when they fit, and flushes its non-zero bins with global FP64 atomics at the end.
#include "common.cuh"
#include "spec.h"

namespace nrg {
namespace {

constexpr int kThreads = 256;

struct Hist {
  double* pos;
  double* neg;
};

// Bins::add (bins.hpp:103-110) + add_std (bins.hpp:112-132) + ChainBinning::add
// (spectrum.hpp:19-24), for a real weight.
NRG_DEV void bin_add(const Hist& h, const BinParams& bp, double energy, double w) {
  if (w == 0.0) return;  // adding an exact zero changes no bin
  double* half = (energy >= 0.0) ? h.pos : h.neg;
  const double e = fabs(energy);
  if (fabs(w) < bp.discard_immediately * e) return;
  if (e < 1e-14) {
    atomicAdd(half, w);
    return;
  }
  const double x = (log10(e) - bp.log10emin) * bp.bins;
  const double ip = floor(x);
  if (ip < 0.0) {
    atomicAdd(half, w);
  } else if (ip >= (double)(bp.nbins - 1)) {
    atomicAdd(half + bp.nbins - 1, w);
  } else {
    const int idx = (int)ip;
    const double rem = x - ip;
    atomicAdd(half + idx, (1.0 - rem) * w);
    atomicAdd(half + idx + 1, rem * w);
  }
}

// The weight of term (i, j) of region r (before `factor`); false for a DM-NRG term outside the
// energy window.
NRG_DEV bool term_weight(const SpecRegion& r, int i, int j, double energy, double& w) {
  const double o1 = r.op1[(int64_t)j * r.ld1 + i];
  switch (r.kind) {
    case kSpecDMNRG: {
      if (fabs(energy) < r.Emin || fabs(energy) > r.Emax) return false;
      const double o2 = r.op2[(int64_t)j * r.ld2 + i];
      const double wA = r.X[(int64_t)j * r.ldx + i] * o1;
      const double wB = r.Y[(int64_t)j * r.ldy + i] * o2;
      w = wA + (double)(-r.sign) * wB;
      return true;
    }
    case kSpecExpI:
      w = o1 * r.op2[(int64_t)j * r.ld2 + i] * r.coef * exp(-r.Ei[i] / r.T);
      return true;
    case kSpecExpJ:
      w = o1 * r.op2[(int64_t)j * r.ld2 + i] * r.coef * exp(-r.Ej[j] / r.T);
      return true;
    default:  // kSpecGemmX
      w = o1 * r.X[(int64_t)j * r.ldx + i] * r.coef;
      return true;
  }
}

__global__ void __launch_bounds__(kThreads) spec_bin_kernel(const SpecTask* __restrict__ tasks,
                                                            const SpecRegion* __restrict__ regs, BinParams bp,
                                                            double* gpos, double* gneg, int use_smem) {
  extern __shared__ __align__(16) double sh[];
  const SpecTask tk = tasks[blockIdx.x];
  const SpecRegion r = regs[tk.region];
  Hist h{gpos, gneg};
  if (use_smem) {
    for (int i = threadIdx.x; i < 2 * bp.nbins; i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
    h.pos = sh;
    h.neg = sh + bp.nbins;
  }
  const int wi = r.i1 - r.i0;
  for (int64_t t = tk.t0 + threadIdx.x; t < tk.t1; t += blockDim.x) {
    const int j = r.j0 + (int)(t / wi);
    const int i = r.i0 + (int)(t % wi);
    const double energy = r.Ej[j] - r.Ei[i];
    double w;
    if (!term_weight(r, i, j, energy, w)) continue;
    bin_add(h, bp, energy, r.factor * w);
  }
  if (use_smem) {
    __syncthreads();
    for (int i = threadIdx.x; i < bp.nbins; i += blockDim.x) {
      if (sh[i] != 0.0) atomicAdd(gpos + i, sh[i]);
      if (sh[bp.nbins + i] != 0.0) atomicAdd(gneg + i, sh[bp.nbins + i]);
    }
  }
}

// Algo_FDMmats, Algo_FTmats, Algo_DMNRGmats (c++/algo_FDM.hpp:167-217, c++/algo_FT.hpp:63-85,
// c++/algo_DMNRG.hpp:76-100) into ChainMatsubara (c++/spectrum.hpp:34-42): every
// term adds factor w / (i w_n - E) = factor w (-E - i w_n) / (E^2 + w_n^2) to point n, for
// n < mats, into a per-CTA copy of the sums in shared memory, flushed with FP64 atomics.
__global__ void __launch_bounds__(kThreads) spec_mats_kernel(const SpecTask* __restrict__ tasks,
                                                             const SpecRegion* __restrict__ regs, MatsParams mp,
                                                             double* gre, double* gim) {
  extern __shared__ __align__(16) double sh[];
  const SpecTask tk = tasks[blockIdx.x];
  const SpecRegion r = regs[tk.region];
  double* re = sh;
  double* im = sh + mp.mats;
  for (int n = threadIdx.x; n < 2 * mp.mats; n += blockDim.x) sh[n] = 0.0;
  __syncthreads();
  const double pt = 3.14159265358979323846 * mp.T;
  const int wi = r.i1 - r.i0;
  for (int64_t t = tk.t0 + threadIdx.x; t < tk.t1; t += blockDim.x) {
    const int j = r.j0 + (int)(t / wi);
    const int i = r.i0 + (int)(t % wi);
    const double energy = r.Ej[j] - r.Ei[i];
    double w;
    if (!term_weight(r, i, j, energy, w)) continue;
    w *= r.factor;
    for (int n = 0; n < mp.mats; n++) {
      if (n == 0 && mp.bosonic && r.mspecial != kMatsPlain && fabs(energy) <= 1e-8) {
        double v = 0.0;
        if (r.mspecial == kMatsMinusOverT) v = -w / mp.T;
        else if (r.mspecial == kMatsPlusOverT) v = w / mp.T;
        else if (r.mspecial == kMatsDmnrgA)
          v = -r.factor * r.X[(int64_t)j * r.ldx + i] * r.op1[(int64_t)j * r.ld1 + i] / mp.T;
        if (v != 0.0) atomicAdd(re, v);
        continue;
      }
      const double wn = pt * (double)(mp.bosonic ? 2 * n : 2 * n + 1);
      const double d = energy * energy + wn * wn;
      atomicAdd(re + n, -w * energy / d);
      atomicAdd(im + n, -w * wn / d);
    }
  }
  __syncthreads();
  for (int n = threadIdx.x; n < mp.mats; n += blockDim.x) {
    if (re[n] != 0.0) atomicAdd(gre + n, re[n]);
    if (im[n] != 0.0) atomicAdd(gim + n, im[n]);
  }
}

}  // namespace

cudaError_t spec_mats_launch(const SpecTask* d_tasks, int ntask, const SpecRegion* d_regs, const MatsParams& mp,
                             double* re, double* im, cudaStream_t stream) {
  if (ntask <= 0 || mp.mats <= 0) return cudaSuccess;
  const size_t smem = 2 * sizeof(double) * (size_t)mp.mats;
  if (smem > kSpecSmemMax) return cudaErrorInvalidValue;
  cudaError_t err =
      cudaFuncSetAttribute(spec_mats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpecSmemMax);
  if (err != cudaSuccess) return err;
  spec_mats_kernel<<<ntask, kThreads, smem, stream>>>(d_tasks, d_regs, mp, re, im);
  return cudaGetLastError();
}

cudaError_t spec_bin_launch(const SpecTask* d_tasks, int ntask, const SpecRegion* d_regs, const BinParams& bp,
                            double* pos, double* neg, cudaStream_t stream) {
  if (ntask <= 0) return cudaSuccess;
  const size_t smem = 2 * sizeof(double) * (size_t)bp.nbins;
  const int use_smem = smem <= kSpecSmemMax ? 1 : 0;
  if (use_smem) {
    cudaError_t err =
        cudaFuncSetAttribute(spec_bin_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpecSmemMax);
    if (err != cudaSuccess) return err;
  }
  spec_bin_kernel<<<ntask, kThreads, use_smem ? smem : 0, stream>>>(d_tasks, d_regs, bp, pos, neg, use_smem);
  return cudaGetLastError();
}

}  // namespace nrg
