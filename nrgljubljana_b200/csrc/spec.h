// spec.h -- internal descriptors of the spectral-weight binning and Matsubara kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nrg {

enum SpecKind : int {
  kSpecDMNRG = 0,  // w = X(j,i) op1(j,i) - sign Y(j,i) op2(j,i), energy window [Emin, Emax]
  kSpecExpI = 1,   // w = coef op1(j,i) op2(j,i) exp(-Ei/T)
  kSpecExpJ = 2,   // w = coef op1(j,i) op2(j,i) exp(-Ej/T)
  kSpecGemmX = 3,  // w = coef op1(j,i) X(j,i)
};

// One rectangle of (i, j) index pairs of one subspace pair with one weight formula.
// The energy of a term is Ej[j] - Ei[i]; every weight is multiplied by `factor`.
struct SpecRegion {
  const double* Ei;
  const double* Ej;
  const double* op1;
  const double* op2;
  const double* X;
  const double* Y;
  int64_t ld1, ld2, ldx, ldy;
  int i0, i1, j0, j1;
  int kind, sign;
  int mspecial, pad_;  // Matsubara sums: a MatsSpecial
  double coef, factor, T, Emin, Emax;
};

// How a term enters the Matsubara sum at n = 0 for a bosonic operator when |E| <= 1e-8
// (WEIGHT_TOL, c++/numerics.hpp:318), where the reference replaces (wA + wB) / (i w_0 - E) by
// a limit: -wA / T for the D x D term of Algo_FDMmats (c++/algo_FDM.hpp:178-188), wA its
// exp(-Ei/T) part (kMatsMinusOverT on that part, kMatsZero on the other); -op1 op2
// exp(-E1/T) / (Z T) for Algo_FTmats (c++/algo_FT.hpp:66-71; kMatsPlusOverT on the
// (-sign) exp(-Ej/T) part, kMatsZero on the other); -wA / T for Algo_DMNRGmats
// (c++/algo_DMNRG.hpp:88-93), wA = X(j,i) op1(j,i) (kMatsDmnrgA).
enum MatsSpecial : int { kMatsPlain = 0, kMatsMinusOverT = 1, kMatsZero = 2, kMatsPlusOverT = 3, kMatsDmnrgA = 4 };

struct MatsParams {
  int mats;     // points n = 0 .. mats-1
  int bosonic;  // w_n = 2 n pi T (bosonic) or (2 n + 1) pi T (fermionic)
  double T;
};

struct SpecTask {  // a contiguous range [t0, t1) of the terms of one region (t = (j-j0)*(i1-i0) + (i-i0))
  int64_t t0, t1;
  int region, pad_;
};

struct BinParams {
  double log10emin;
  double discard_immediately;
  int bins;   // bins per decade
  int nbins;  // points per sign half
};

constexpr size_t kSpecSmemMax = 96 * 1024;  // private histograms up to 6144 bins per half

cudaError_t spec_bin_launch(const SpecTask* d_tasks, int ntask, const SpecRegion* d_regs, const BinParams& bp,
                            double* pos, double* neg, cudaStream_t stream);
// Matsubara sums: re[n] + i im[n] += factor w / (i w_n - E) for every term (accumulated).
cudaError_t spec_mats_launch(const SpecTask* d_tasks, int ntask, const SpecRegion* d_regs, const MatsParams& mp,
                             double* re, double* im, cudaStream_t stream);

}  // namespace nrg
