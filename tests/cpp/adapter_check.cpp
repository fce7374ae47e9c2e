// Exercises include/nrg_b200.hpp, the header-only C++ adapter with the reference's
// signatures, the way the reference's host code would call it. Prints one line per check
// and "ADAPTER OK" at the end; the exit status is the number of failed checks.
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "nrg_b200.hpp"

using nrg_b200::Matrix;

static int fails = 0;
static void expect(bool ok, const std::string& what) {
  std::printf("%s %s\n", ok ? "ok  " : "FAIL", what.c_str());
  fails += ok ? 0 : 1;
}

static Matrix random_upper(std::mt19937_64& g, std::size_t n) {
  std::normal_distribution<double> nd;
  Matrix m(n, n);
  for (std::size_t i = 0; i < n; i++)
    for (std::size_t j = i; j < n; j++) m(i, j) = nd(g);
  return m;
}

static Matrix random_matrix(std::mt19937_64& g, std::size_t r, std::size_t c) {
  std::normal_distribution<double> nd;
  Matrix m(r, c);
  for (std::size_t i = 0; i < r; i++)
    for (std::size_t j = 0; j < c; j++) m(i, j) = nd(g);
  return m;
}

static double sym(const Matrix& m, std::size_t i, std::size_t j) { return i <= j ? m(i, j) : m(j, i); }

int main() {
  // 1. The 2x2 known-answer cases of the reference's diag unit test
  //    (test/unit/diag_test/diag_test.cpp): sigma_x and sigma_z, upper triangles.
  {
    Matrix sx(2, 2);
    sx(0, 1) = 1.0;
    nrg_b200::DiagParams DP;
    auto d = nrg_b200::diagonalise(sx, DP, 0);
    const double r = 1.0 / std::sqrt(2.0);
    bool ok = d.getnrcomputed() == 2 && std::abs(d.val[0] + 1.0) < 1e-15 && std::abs(d.val[1] - 1.0) < 1e-15;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) ok = ok && std::abs(std::abs(d.vec(i, j)) - r) < 1e-15;
    ok = ok && d.vec(0, 0) * d.vec(0, 1) < 0 && d.vec(1, 0) * d.vec(1, 1) > 0;
    expect(ok, "sigma_x: eigenvalues -1, 1 and |v| = 1/sqrt(2)");
    Matrix sz(2, 2);
    sz(0, 0) = 1.0;
    sz(1, 1) = -1.0;
    DP.diag = "dsyevd";
    auto e = nrg_b200::diagonalise(sz, DP, 0);
    expect(e.val[0] == -1.0 && e.val[1] == 1.0 && std::abs(std::abs(e.vec(0, 1)) - 1.0) < 1e-15,
           "sigma_z (dsyevd): eigenvalues -1, 1, vectors the unit vectors");
  }
  // 2. One batched call for a step's worth of blocks; residuals and orthogonality.
  {
    std::mt19937_64 g(7);
    std::vector<Matrix> blocks;
    for (std::size_t n : {1, 2, 5, 17, 64, 65, 100, 230, 301}) blocks.push_back(random_upper(g, n));
    auto res = nrg_b200::diagonalisations(blocks);
    double worst = 0.0, worst_o = 0.0;
    bool sorted = true;
    for (std::size_t b = 0; b < blocks.size(); b++) {
      const std::size_t n = blocks[b].size1();
      double nrm = 0.0;
      for (double v : res[b].val) nrm = std::max(nrm, std::abs(v));
      for (std::size_t r = 0; r < n; r++) {
        if (r && res[b].val[r] < res[b].val[r - 1]) sorted = false;
        double rr = 0.0;
        for (std::size_t i = 0; i < n; i++) {
          double s = 0.0;
          for (std::size_t j = 0; j < n; j++) s += sym(blocks[b], i, j) * res[b].vec(r, j);
          rr = std::max(rr, std::abs(s - res[b].val[r] * res[b].vec(r, i)));
        }
        worst = std::max(worst, rr / std::max(nrm, 1e-300));
        for (std::size_t q = 0; q <= r; q++) {
          double s = 0.0;
          for (std::size_t i = 0; i < n; i++) s += res[b].vec(r, i) * res[b].vec(q, i);
          worst_o = std::max(worst_o, std::abs(s - (q == r ? 1.0 : 0.0)));
        }
      }
    }
    char buf[160];
    std::snprintf(buf, sizeof buf, "batched diagonalisations: residual %.2e, orthogonality %.2e", worst, worst_o);
    expect(sorted && worst < 1e-12 && worst_o < 1e-12, buf);
    nrg_b200::DiagParams DP;
    DP.diag = "dsyevr";
    DP.diagratio = 0.5;
    auto part = nrg_b200::diagonalise(blocks[6], DP, 0);
    expect(part.getnrcomputed() == 50 && part.vec.size1() == 50 && part.vec.size2() == 100 &&
               part.val[0] == res[6].val[0] && part.val[49] == res[6].val[49],
           "dsyevr with diagratio 0.5: the lowest ceil(0.5 dim) pairs");
  }
  // 3. product / transform / rotate against plain loops.
  {
    std::mt19937_64 g(11);
    const std::size_t r = 13, c = 9, k = 7;
    Matrix A = random_matrix(g, r, k), B = random_matrix(g, c, k), O = random_matrix(g, k, k);
    Matrix M0 = random_matrix(g, r, c);
    Matrix M = M0, P = M0;
    nrg_b200::transform(M, 0.75, A, O, B);
    nrg_b200::product(P, -1.25, A, B);
    double et = 0.0, ep = 0.0;
    for (std::size_t i = 0; i < r; i++)
      for (std::size_t j = 0; j < c; j++) {
        double t = 0.0, p = 0.0;
        for (std::size_t a = 0; a < k; a++) {
          p += A(i, a) * B(j, a);
          for (std::size_t b = 0; b < k; b++) t += A(i, a) * O(a, b) * B(j, b);
        }
        et = std::max(et, std::abs(M(i, j) - (M0(i, j) + 0.75 * t)));
        ep = std::max(ep, std::abs(P(i, j) - (M0(i, j) - 1.25 * p)));
      }
    expect(et < 1e-12 && ep < 1e-12, "transform and product equal the plain loops");
    const std::size_t n = 6, dim = 10;
    Matrix U = random_matrix(g, n, dim), R = random_matrix(g, n, n), D(dim, dim);
    nrg_b200::rotate(D, 2.0, U, R);
    double er = 0.0;
    for (std::size_t i = 0; i < dim; i++)
      for (std::size_t j = 0; j < dim; j++) {
        double s = 0.0;
        for (std::size_t a = 0; a < n; a++)
          for (std::size_t b = 0; b < n; b++) s += U(a, i) * R(a, b) * U(b, j);
        er = std::max(er, std::abs(D(i, j) - 2.0 * s));
      }
    expect(er < 1e-12, "rotate equals U^T O U");
  }
  // 4. Errors as the reference raises them.
  {
    Matrix m(3, 3), a(3, 2), b(3, 2), o(2, 2);
    bool thrown = false;
    try {
      nrg_b200::transform(m, std::nan(""), a, o, b);
    } catch (const nrg_b200::Error& e) {
      thrown = e.code() == NRG_ERR_ARG;
    }
    expect(thrown, "a non-finite factor is rejected (my_assert(my_isfinite(factor)))");
    Matrix bad(3, 3);
    bad(0, 0) = std::nan("");
    std::string msg;
    try {
      nrg_b200::diagonalise(bad, nrg_b200::DiagParams(), 0);
    } catch (const std::runtime_error& e) {
      msg = e.what();
    }
    expect(msg.rfind("dsyev failed. INFO=", 0) == 0, "a failed block throws \"dsyev failed. INFO=...\": " + msg);
    Matrix low(2, 2);
    low(1, 0) = 1.0;
    thrown = false;
    try {
      nrg_b200::diagonalise(low, nrg_b200::DiagParams(), 0);
    } catch (const std::invalid_argument&) {
      thrown = true;
    }
    expect(thrown, "a non-zero lower triangle is rejected (is_matrix_upper)");
    Matrix wrong(4, 3);
    thrown = false;
    try {
      nrg_b200::product(wrong, 1.0, a, b);
    } catch (const std::invalid_argument&) {
      thrown = true;
    }
    expect(thrown, "non-conforming shapes are rejected");
  }
  std::printf("%s\n", fails ? "ADAPTER FAILED" : "ADAPTER OK");
  return fails;
}
