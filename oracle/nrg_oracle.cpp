// nrg_oracle.cpp -- CPU oracle for the NRG step core.
//
// TEST INFRASTRUCTURE ONLY. This file restates, on the CPU and in plain C++ over the
// host LAPACK/BLAS (the OpenBLAS that ships with scipy, LP64, symbols prefixed
// `scipy_`), the reference algorithms of NRG Ljubljana 2020.10 for the hot path:
//   * block diagonalisation            c++/diag.hpp:62-82 (dsyev), 85-115 (dsyevd), 118-172 (dsyevr)
//   * eigenvector unitarity check      c++/numerics.hpp:340-367, 399-404
//   * GEMM leaves                      c++/numerics_ublas.hpp:108-140 (product, transform, rotate)
//   * prod_fit                         c++/numerics.hpp:283-306
//   * log-grid binning                 c++/bins.hpp:61-69, 95-132; c++/spectrum.hpp:19-28
//   * N/N+2 window merge               c++/spectrum.hpp:91-128
//   * DM-NRG spectral weights          c++/algo_DMNRG.hpp:29-52
//   * FDM spectral weights             c++/algo_FDM.hpp:30-60 (ls), 84-114 (gt)
//   * chit_weight                      c++/numerics.hpp:308-327
// Only the test-suite, the smoke check and the CPU-baseline leg of the benchmark load
// it, always as the checker or as the timed CPU reference; the product path never does.
//
// Layout conventions are the reference's: matrices are dense row-major; a diagonalised
// block returns ascending eigenvalues and eigenvectors as ROWS (vec(r, j)).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
void scipy_dsyev_(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w, double* work,
                  const int* lwork, int* info);
void scipy_dsyevd_(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w, double* work,
                   const int* lwork, int* iwork, const int* liwork, int* info);
void scipy_dsyevr_(const char* jobz, const char* range, const char* uplo, const int* n, double* a, const int* lda,
                   const double* vl, const double* vu, const int* il, const int* iu, const double* abstol, int* m,
                   double* w, double* z, const int* ldz, int* isuppz, double* work, const int* lwork, int* iwork,
                   const int* liwork, int* info);
void scipy_dgemm_(const char* transa, const char* transb, const int* m, const int* n, const int* k,
                  const double* alpha, const double* a, const int* lda, const double* b, const int* ldb,
                  const double* beta, double* c, const int* ldc);
void scipy_openblas_set_num_threads(int);
int scipy_openblas_get_num_threads(void);
}

namespace {

// Row-major C(m x n) = alpha * op(A) * op(B) + beta * C, mapped onto column-major dgemm by
// computing C^T = op(B)^T op(A)^T.
void gemm_rm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb,
             double beta, double* C, int ldc) {
  if (m == 0 || n == 0) return;
  const char TA = tb ? 'T' : 'N';
  const char TB = ta ? 'T' : 'N';
  scipy_dgemm_(&TA, &TB, &n, &m, &k, &alpha, B, &ldb, A, &lda, &beta, C, &ldc);
}

// diag.hpp:62-82. The row-major matrix with its upper triangle set is handed to LAPACK
// with UPLO='L' (column-major lower == row-major upper). Column-major Z read as a
// row-major matrix has eigenvector r in row r (diag.hpp:41-48).
int dsyev_one(int n, double* H, double* w) {
  const char jobz = 'V', uplo = 'L';
  int info = 0, lwork = -1;
  double wq = 0;
  scipy_dsyev_(&jobz, &uplo, &n, H, &n, w, &wq, &lwork, &info);
  if (info != 0) return info;
  lwork = int(wq);
  std::vector<double> work(std::max(1, lwork));
  scipy_dsyev_(&jobz, &uplo, &n, H, &n, w, work.data(), &lwork, &info);
  return info;
}

// diag.hpp:85-115
int dsyevd_one(int n, double* H, double* w) {
  const char jobz = 'V', uplo = 'L';
  int info = 0, lwork = -1, liwork = -1, iwq = 0;
  double wq = 0;
  scipy_dsyevd_(&jobz, &uplo, &n, H, &n, w, &wq, &lwork, &iwq, &liwork, &info);
  if (info != 0) return info;
  lwork = int(wq);
  liwork = iwq;
  std::vector<double> work(std::max(1, lwork));
  std::vector<int> iwork(std::max(1, liwork));
  scipy_dsyevd_(&jobz, &uplo, &n, H, &n, w, work.data(), &lwork, iwork.data(), &liwork, &info);
  return info;
}

// diag.hpp:118-172 (RANGE='I' when ratio != 1; returns the number of computed pairs in *m).
int dsyevr_one(int n, double* H, double* w, double* Z, double ratio, int* mout) {
  const char jobz = 'V', uplo = 'L';
  char range = 'A';
  int M = n;
  if (ratio != 1.0) {
    M = int(std::ceil(ratio * n));
    M = std::clamp(M, 1, n);
    range = 'I';
  }
  const double vl = 0, vu = 0, abstol = 0;
  int il = 1, iu = M, mm = 0, info = 0, lwork = -1, liwork = -1, iwq = 0;
  double wq = 0;
  std::vector<int> isuppz(2 * std::max(1, M));
  scipy_dsyevr_(&jobz, &range, &uplo, &n, H, &n, &vl, &vu, &il, &iu, &abstol, &mm, w, Z, &n, isuppz.data(), &wq,
                &lwork, &iwq, &liwork, &info);
  if (info != 0) return info;
  lwork = int(wq);
  liwork = iwq;
  std::vector<double> work(std::max(1, lwork));
  std::vector<int> iwork(std::max(1, liwork));
  scipy_dsyevr_(&jobz, &range, &uplo, &n, H, &n, &vl, &vu, &il, &iu, &abstol, &mm, w, Z, &n, isuppz.data(),
                work.data(), &lwork, iwork.data(), &liwork, &info);
  *mout = mm;
  return info;
}

// numerics.hpp:107-114 (my_fcmp) and 118-120 (num_equal)
bool num_equal(double x, double y, double eps) {
  if (x == 0.0 && y == 0.0) return true;
  if (std::abs(x) < eps && std::abs(y) < eps) return true;
  return std::abs(x - y) < eps * (std::abs(x) + std::abs(y));
}

}  // namespace

extern "C" {

int oracle_blas_threads(int n) {
  if (n > 0) scipy_openblas_set_num_threads(n);
  return scipy_openblas_get_num_threads();
}

// One block: H (n x n, row-major, upper triangle read, destroyed); evals[n] ascending;
// evecs (n x n row-major, row r = eigenvector r). solver: 0 dsyev, 1 dsyevd (falls back
// to dsyev on INFO>0 as diag.hpp:269-275), 2 dsyevr with `ratio` (diag.hpp:276).
// Returns LAPACK INFO; *mout receives the number of computed pairs.
int oracle_diagonalise(int n, double* H, double* evals, double* evecs, int solver, double ratio, int* mout) {
  if (n <= 0) return -1;
  int info = 0;
  *mout = n;
  if (solver == 2) {
    info = dsyevr_one(n, H, evals, evecs, ratio, mout);
    return info;
  }
  std::vector<double> backup;
  if (solver == 1) {
    backup.assign(H, H + size_t(n) * n);
    info = dsyevd_one(n, H, evals);
    if (info > 0) {  // diag.hpp:106-110 + 269-274
      std::copy(backup.begin(), backup.end(), H);
      info = dsyev_one(n, H, evals);
    }
  } else {
    info = dsyev_one(n, H, evals);
  }
  if (info == 0) std::memcpy(evecs, H, sizeof(double) * size_t(n) * n);
  return info;
}

// The batch loop of core.hpp:90-110 (OpenMP over blocks, schedule(dynamic), BLAS threads
// set by the caller). Blocks are packed: block b starts at mat_off[b] (n_b*n_b doubles) in
// H/evecs and at val_off[b] in evals. Blocks are visited in decreasing size order
// (TaskList, subspaces.hpp:114-121). Returns the number of blocks with INFO != 0.
int oracle_diag_batch(int nblk, const int* n, const int64_t* mat_off, const int64_t* val_off, double* H,
                      double* evals, double* evecs, int solver, int nthreads, int* info_out) {
  std::vector<int> order(nblk);
  for (int i = 0; i < nblk; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [n](int a, int b) { return n[a] > n[b]; });
  int nbad = 0;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads) reduction(+ : nbad)
  for (int t = 0; t < nblk; t++) {
    const int b = order[t];
    int m = 0;
    const int info = oracle_diagonalise(n[b], H + mat_off[b], evals + val_off[b], evecs + mat_off[b], solver, 1.0, &m);
    info_out[b] = info;
    if (info != 0) nbad++;
  }
  return nbad;
}

// numerics.hpp:340-367: 1 if the M rows of vec (M x dim) are orthonormal.
int oracle_is_unitary(int M, int dim, const double* vec, double norm_eps, double ortho_eps) {
  for (int r = 0; r < M; r++) {
    double s = 0;
    for (int j = 0; j < dim; j++) s += vec[size_t(r) * dim + j] * vec[size_t(r) * dim + j];
    if (!num_equal(std::abs(s), 1.0, norm_eps)) return 0;
  }
  for (int r1 = 0; r1 < M; r1++)
    for (int r2 = r1 + 1; r2 < M; r2++) {
      double s = 0;
      for (int j = 0; j < dim; j++) s += vec[size_t(r1) * dim + j] * vec[size_t(r2) * dim + j];
      if (!num_equal(std::abs(s), 0.0, ortho_eps)) return 0;
    }
  return 1;
}

// numerics_ublas.hpp:108-116. M (m x n) += factor * A (m x k) * B^T, B is n x k.
// Leading dimensions allow strided views such as U(i) blocks (recalc.hpp:18-30).
void oracle_product(int m, int n, int k, double factor, const double* A, int lda, const double* B, int ldb, double* M,
                    int ldm) {
  if (m == 0 || n == 0 || k == 0) return;
  gemm_rm(false, true, m, n, k, factor, A, lda, B, ldb, 1.0, M, ldm);
}

// numerics_ublas.hpp:119-128. M (m x n) += factor * A (m x ka) * O (ka x kb) * B^T, B is n x kb.
// Same association as the reference: T = O * B^T first, then M += factor * A * T.
void oracle_transform(int m, int n, int ka, int kb, double factor, const double* A, int lda, const double* O, int ldo,
                      const double* B, int ldb, double* M, int ldm) {
  if (m == 0 || n == 0 || ka == 0 || kb == 0) return;
  std::vector<double> T(size_t(ka) * n);
  gemm_rm(false, true, ka, n, kb, 1.0, O, ldo, B, ldb, 0.0, T.data(), n);
  gemm_rm(false, false, m, n, ka, factor, A, lda, T.data(), n, 1.0, M, ldm);
}

// numerics_ublas.hpp:130-140. M (d x d) += factor * U^T * O * U, U is k x d, O is k x k.
void oracle_rotate(int d, int k, double factor, const double* U, int ldu, const double* O, int ldo, double* M, int ldm) {
  if (d == 0 || k == 0) return;
  std::vector<double> T(size_t(d) * k);
  gemm_rm(true, false, d, k, k, 1.0, U, ldu, O, ldo, 0.0, T.data(), k);
  gemm_rm(false, false, d, d, k, factor, T.data(), k, U, ldu, 1.0, M, ldm);
}

// Plain C = A * B (numerics_ublas.hpp:154-161, matrix_prod), used by prod_fit.
void oracle_matmul(int m, int n, int k, const double* A, int lda, const double* B, int ldb, double* C, int ldc) {
  gemm_rm(false, false, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, ldc);
}

// numerics.hpp:308-327
double oracle_chit_weight(double En, double Em, double beta) {
  const double betaEn = beta * En, betaEm = beta * Em, x = betaEn - betaEm;
  if (std::abs(x) > 1e-8) return (std::exp(-betaEm) - std::exp(-betaEn)) / x;
  return std::exp(-betaEm);
}

// ---------------------------------------------------------------- binning
// bins.hpp:95-100 (loggrid_std) with setlimits 61-69 folded into (log10emin, log10emax).
// Returns the number of bins; fills energies[] if non-null.
int oracle_loggrid(double log10emin, double log10emax, int bins, double* energies) {
  const int nr = int((log10emax - log10emin) * bins + 1.0);
  if (energies)
    for (int i = 0; i < nr; i++) energies[i] = std::pow(10.0, log10emin + double(i) / bins);
  return nr;
}

// bins.hpp:103-132 (add + add_std) for one sign half; w is the (re, im) weight pair.
static inline void bins_add_std(double* wre, double* wim, int nbins, double log10emin, int bins, double energy,
                                double are, double aim, double discard_immediately) {
  if (std::abs(std::complex<double>(are, aim)) < discard_immediately * energy) return;
  if (energy < 1e-14) {
    wre[0] += are;
    wim[0] += aim;
    return;
  }
  const double x = (std::log10(energy) - log10emin) * bins;
  const double ip = std::floor(x);
  if (ip < 0) {
    wre[0] += are;
    wim[0] += aim;
  } else if (size_t(ip) >= size_t(nbins - 1)) {
    wre[nbins - 1] += are;
    wim[nbins - 1] += aim;
  } else {
    const size_t idx = size_t(ip);
    const double rem = x - ip;
    wre[idx] += (1.0 - rem) * are;
    wim[idx] += (1.0 - rem) * aim;
    wre[idx + 1] += rem * are;
    wim[idx + 1] += rem * aim;
  }
}

// ChainBinning::add (spectrum.hpp:19-28): non-negative energies go to the positive half,
// negative ones (sign flipped) to the negative half. Arrays hold nbins doubles each.
void oracle_chain_add(double* pos_re, double* pos_im, double* neg_re, double* neg_im, int nbins, double log10emin,
                      int bins, double discard_immediately, int nterm, const double* energy, const double* wre,
                      const double* wim, double factor) {
  for (int t = 0; t < nterm; t++) {
    const double e = energy[t];
    const double are = factor * wre[t], aim = factor * (wim ? wim[t] : 0.0);
    if (e >= 0.0)
      bins_add_std(pos_re, pos_im, nbins, log10emin, bins, e, are, aim, discard_immediately);
    else
      bins_add_std(neg_re, neg_im, nbins, log10emin, bins, -e, are, aim, discard_immediately);
  }
}

// spectrum.hpp:91-109, windowfunction. flags: bit0 step.last(), bit1 step.first(), bit2 ZBW.
double oracle_windowfunction(double E, double Emin, double Ex, double Emax, int flags, double NNtanh) {
  if (E <= Ex && (flags & 1)) return 1.0;
  if (E >= Ex && (flags & 2)) return 1.0;
  if (flags & 4) return 1.0;
  if (E <= Emin || E >= Emax) return 0.0;
  auto lin = [](double x) { return x; };
  auto th0 = [](double x, double a) { return std::tanh(a * (x - 0.5)); };
  auto th = [&](double x, double a) { return (th0(x, a) - th0(0, a)) / (th0(1, a) - th0(0, a)); };
  auto fnc = [&](double x) { return NNtanh > 0 ? th(x, NNtanh) : lin(x); };
  if (Emin < E && E <= Ex) return fnc((E - Emin) / (Ex - Emin));
  if (Ex < E && E < Emax) return 1.0 - fnc((E - Ex) / (Emax - Ex));
  return 0.0;
}

// spectrum.hpp:114-128, mergeNN2half for one sign half.
void oracle_merge_nn2half(double* full_re, double* full_im, const double* cs_re, const double* cs_im,
                          const double* energies, int nbins, double Emin, double Ex, double Emax, int flags,
                          double NNtanh, int NN2avg) {
  for (int i = 0; i < nbins; i++) {
    const double e = energies[i];
    if (Emin < e && e < Emax && (cs_re[i] != 0.0 || cs_im[i] != 0.0)) {
      const double f = (NN2avg ? 0.5 : 1.0) * oracle_windowfunction(e, Emin, Ex, Emax, flags, NNtanh);
      full_re[i] += f * cs_re[i];
      full_im[i] += f * cs_im[i];
    }
  }
}

// algo_DMNRG.hpp:29-52 for one subspace pair (Ip, I1). op1, op2: dim1 x dimp (rows: I1
// states, cols: Ip states), row-major with leading dimensions. rhoP (ldrp) and rho1
// (ldr1) are the density matrices of Ip and I1. Em/Ej are abs_zero energies. Only kept
// states enter (kp, k1). Weights are real (S = double) and accumulated into the chain
// binning arrays with `factor` exactly as the triple loop does.
void oracle_dmnrg_pair(int kp, int k1, const double* Em, const double* Ej, const double* op1, int ld1,
                       const double* op2, int ld2, const double* rhoP, int ldrp, const double* rho1, int ldr1,
                       double factor, int sign, double Emin, double Emax, double* pos_re, double* pos_im,
                       double* neg_re, double* neg_im, int nbins, double log10emin, int bins,
                       double discard_immediately) {
  for (int rm = 0; rm < kp; rm++)
    for (int rj = 0; rj < k1; rj++) {
      const double energy = Ej[rj] - Em[rm];
      double wA = 0, wB = 0;
      if (!(std::abs(energy) < Emin || std::abs(energy) > Emax)) {
        double sumA = 0;
        for (int ri = 0; ri < kp; ri++) sumA += op2[size_t(rj) * ld2 + ri] * rhoP[size_t(rm) * ldrp + ri];
        wA = sumA * op1[size_t(rj) * ld1 + rm];
        double sumB = 0;
        for (int ri = 0; ri < k1; ri++) sumB += op1[size_t(ri) * ld1 + rm] * rho1[size_t(rj) * ldr1 + ri];
        wB = sumB * op2[size_t(rj) * ld2 + rm];
      }
      const double w = wA + (-sign) * wB;
      const double zero = 0.0;
      oracle_chain_add(pos_re, pos_im, neg_re, neg_im, nbins, log10emin, bins, discard_immediately, 1, &energy, &w,
                       &zero, factor);
    }
}

// algo_FDM.hpp:84-114 (gt, which=0) and 30-60 (ls, which=1) for one pair (Ii, Ij).
// op1, op2: dimj x dimi. Ei/Ej are abs_G energies of all stored states; [0, Ki) / [0, Kj)
// are the kept ranges (Krange), [Ki, ni) / [Kj, nj) the discarded ones (Drange).
// rho: rhoFDM(Ii) (ni x ni) for gt, rhoFDM(Ij) (nj x nj) for ls.
// prod_fit (numerics.hpp:283-306) restated for these shapes.
void oracle_fdm_pair(int which, int ni, int Ki, int nj, int Kj, const double* Ei, const double* Ej, const double* op1,
                     int ld1, const double* op2, int ld2, const double* rho, int ldr, int rho_dim, double factor,
                     int sign, double T, double wnf, double* pos_re, double* pos_im, double* neg_re, double* neg_im,
                     int nbins, double log10emin, int bins, double discard_immediately) {
  auto add = [&](double e, double w) {
    const double z = 0.0;
    oracle_chain_add(pos_re, pos_im, neg_re, neg_im, nbins, log10emin, bins, discard_immediately, 1, &e, &w, &z,
                     factor);
  };
  if (which == 0) {
    // op2_rho = prod_fit(op2, rho(Ii)): op2 is nj x ni, rho is rho_dim x rho_dim; the
    // product is nj x rho_dim. prod_fit_left (rho_dim <= ni) uses op2[:, :rho_dim] * rho,
    // prod_fit_right uses op2 * rho[:ni, :].
    const int outc = rho_dim;
    std::vector<double> X(size_t(nj) * outc, 0.0);
    if (rho_dim <= ni)
      gemm_rm(false, false, nj, rho_dim, rho_dim, 1.0, op2, ld2, rho, ldr, 0.0, X.data(), outc);
    else
      gemm_rm(false, false, nj, rho_dim, ni, 1.0, op2, ld2, rho, ldr, 0.0, X.data(), outc);
    for (int i = Ki; i < ni; i++)
      for (int j = Kj; j < nj; j++)
        add(Ej[j] - Ei[i], op1[size_t(j) * ld1 + i] * op2[size_t(j) * ld2 + i] * std::exp(-Ei[i] / T) * wnf);
    for (int i = Ki; i < ni; i++)
      for (int j = 0; j < Kj; j++)
        add(Ej[j] - Ei[i], op1[size_t(j) * ld1 + i] * op2[size_t(j) * ld2 + i] * std::exp(-Ei[i] / T) * wnf);
    for (int i = 0; i < Ki; i++)
      for (int j = Kj; j < nj; j++) add(Ej[j] - Ei[i], op1[size_t(j) * ld1 + i] * X[size_t(j) * outc + i]);
  } else {
    // rho_op2 = prod_fit(rho(Ij), op2): rho is rho_dim x rho_dim, op2 is nj x ni.
    const int outc = ni;
    std::vector<double> X(size_t(rho_dim) * outc, 0.0);
    if (nj <= rho_dim)  // prod_fit_left: rho[:, :nj] * op2 -> rho_dim x ni
      gemm_rm(false, false, rho_dim, ni, nj, 1.0, rho, ldr, op2, ld2, 0.0, X.data(), outc);
    else  // prod_fit_right: rho * op2[:rho_dim, :]
      gemm_rm(false, false, rho_dim, ni, rho_dim, 1.0, rho, ldr, op2, ld2, 0.0, X.data(), outc);
    for (int i = Ki; i < ni; i++)
      for (int j = Kj; j < nj; j++)
        add(Ej[j] - Ei[i], op1[size_t(j) * ld1 + i] * op2[size_t(j) * ld2 + i] * (-sign) * std::exp(-Ej[j] / T) * wnf);
    for (int i = Ki; i < ni; i++)
      for (int j = 0; j < Kj; j++) add(Ej[j] - Ei[i], op1[size_t(j) * ld1 + i] * X[size_t(j) * outc + i] * (-sign));
    for (int i = 0; i < Ki; i++)
      for (int j = Kj; j < nj; j++)
        add(Ej[j] - Ei[i], op1[size_t(j) * ld1 + i] * op2[size_t(j) * ld2 + i] * (-sign) * std::exp(-Ej[j] / T) * wnf);
  }
}

}  // extern "C"
