/* nrg_b200.hpp -- header-only C++ adapter of the B200 NRG step core with the signatures of
 * NRG Ljubljana's host code, over the C-ABI of nrg_b200.h.
 *
 * A maintainer of the reference binds the GPU path by calling these in place of the CPU
 * routines they are named after; the argument order, the in-place accumulation and the
 * exceptions are the reference's:
 *
 *   diagonalise(m, DP, myrank)           c++/diag.hpp:261-292   (real matrices)
 *   diagonalisations(blocks, DP)         c++/core.hpp:90-120    (one batched call per step)
 *   product(M, factor, A, B)             c++/numerics_ublas.hpp:108-116   M += f A B^T
 *   transform(M, factor, A, O, B)        c++/numerics_ublas.hpp:119-128   M += f A O B^T
 *   rotate(M, factor, U, O)              c++/numerics_ublas.hpp:130-140   M += f U^T O U
 *
 * Matrix types: any M with size1(), size2(), element access m(i, j) returning a reference
 * and contiguous row-major storage whose first element is &m(0, 0) (leading dimension
 * size2()): boost::numeric::ublas::matrix<double> (row_major, unbounded_array) qualifies,
 * and so does nrg_b200::Matrix below, a minimal stand-in for builds without Boost. Host
 * matrices go through the _host entry points (copy in, compute on the GPU, copy out).
 *
 * Errors: a LAPACK-style failure of a block (its status word != 0) throws
 * std::runtime_error("dsyev failed. INFO=<info>"), as c++/diag.hpp:80 does; shape
 * mismatches (the reference's my_assert) throw std::invalid_argument; a failure of the
 * library (no sm_100 device, out of memory, invalid argument such as a non-finite factor)
 * throws nrg_b200::Error with the library's message. Nothing falls back to the CPU.
 *
 * Contexts: one per host thread and device (thread_local), created at first use and
 * destroyed when the thread exits, so concurrent callers (the reference's OpenMP worker
 * threads, c++/core.hpp:98-107) never share one.
 */
#ifndef NRG_B200_HPP
#define NRG_B200_HPP

#include <cmath>
#include <cstddef>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "nrg_b200.h"

namespace nrg_b200 {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* where) {
  if (rc < 0) throw Error(rc, std::string(where) + ": " + nrg_last_error());
}

// Minimal dense row-major matrix with the ublas accessors the adapter uses.
class Matrix {
 public:
  using value_type = double;
  Matrix() = default;
  Matrix(std::size_t r, std::size_t c, double v = 0.0) : r_(r), c_(c), a_(r * c, v) {}
  std::size_t size1() const { return r_; }
  std::size_t size2() const { return c_; }
  double& operator()(std::size_t i, std::size_t j) { return a_[i * c_ + j]; }
  const double& operator()(std::size_t i, std::size_t j) const { return a_[i * c_ + j]; }
  double* data() { return a_.data(); }
  const double* data() const { return a_.data(); }

 private:
  std::size_t r_ = 0, c_ = 0;
  std::vector<double> a_;
};

// The reference's DiagParams (c++/params.hpp:664-676): solver name and, for dsyevr, the
// fraction of the spectrum to return.
struct DiagParams {
  std::string diag = "default";
  double diagratio = 1.0;
};

// Eigenvalues ascending and eigenvectors as rows (c++/eigen.hpp:180-199).
template <class M>
struct RawEigen {
  std::vector<double> val;
  M vec;
  std::size_t getnrcomputed() const { return val.size(); }
  std::size_t getdim() const { return vec.size2(); }
};

namespace detail {

template <class M>
const double* base(const M& m) {
  return (m.size1() && m.size2()) ? &m(0, 0) : nullptr;
}
template <class M>
double* base(M& m) {
  return (m.size1() && m.size2()) ? &m(0, 0) : nullptr;
}

struct ThreadContexts {
  std::map<int, nrg_ctx*> ctx;
  ~ThreadContexts() {
    for (auto& kv : ctx) nrg_destroy(kv.second);
  }
};

inline nrg_ctx* context(int device) {
  thread_local ThreadContexts tc;
  auto it = tc.ctx.find(device);
  if (it != tc.ctx.end()) return it->second;
  nrg_ctx* c = nullptr;
  check(nrg_create(&c, device, 0), "nrg_create");
  tc.ctx[device] = c;
  return c;
}

// c++/numerics.hpp:140-146: square, strictly lower triangle zero.
template <class M>
bool is_matrix_upper(const M& m) {
  if (m.size1() != m.size2()) return false;
  for (std::size_t i = 1; i < m.size1(); i++)
    for (std::size_t j = 0; j < i; j++)
      if (std::abs(m(i, j)) >= 1e-12) return false;
  return true;
}

// Number of eigenpairs the reference returns: all, or for dsyevr the lowest
// ceil(diagratio * dim) (c++/diag.hpp:118-130).
inline std::size_t nr_returned(const DiagParams& DP, std::size_t dim) {
  if (DP.diag == "dsyevr" && DP.diagratio < 1.0) {
    const std::size_t m = static_cast<std::size_t>(std::ceil(DP.diagratio * static_cast<double>(dim)));
    return m < 1 ? 1 : (m > dim ? dim : m);
  }
  return dim;
}

inline void check_solver(const DiagParams& DP) {
  if (DP.diag != "default" && DP.diag != "dsyev" && DP.diag != "dsyevd" && DP.diag != "dsyevr")
    throw std::invalid_argument("diag=" + DP.diag + ": the GPU path solves real symmetric blocks only");
}

}  // namespace detail

// The device this thread's calls use (default 0).
inline int& current_device() {
  thread_local int dev = 0;
  return dev;
}

// All blocks of one step in one batched call; blocks[b] is square with its upper triangle
// set (the lower triangle must be zero, as c++/diag.hpp:265 asserts) and is left unchanged.
template <class M>
std::vector<RawEigen<M>> diagonalisations(const std::vector<M>& blocks, const DiagParams& DP = DiagParams()) {
  detail::check_solver(DP);
  const std::size_t nb = blocks.size();
  std::vector<RawEigen<M>> out(nb);
  if (nb == 0) return out;
  std::vector<int> n(nb), info(nb, 0);
  std::vector<const double*> H(nb);
  std::vector<std::vector<double>> val(nb);
  std::vector<M> vec;
  vec.reserve(nb);
  std::vector<double*> pv(nb), pz(nb);
  for (std::size_t b = 0; b < nb; b++) {
    const M& m = blocks[b];
    if (!detail::is_matrix_upper(m)) throw std::invalid_argument("is_matrix_upper(m) failed");
    if (m.size1() == 0) throw std::invalid_argument("empty block");
    n[b] = static_cast<int>(m.size1());
    H[b] = detail::base(m);
    val[b].resize(m.size1());
    vec.emplace_back(m.size1(), m.size1());
    pv[b] = val[b].data();
    pz[b] = detail::base(vec[b]);
  }
  const int rc = nrg_diag_batch_host(detail::context(current_device()), static_cast<int>(nb), n.data(), H.data(),
                                     pv.data(), pz.data(), info.data(), nullptr);
  check(rc, "nrg_diag_batch_host");
  for (std::size_t b = 0; b < nb; b++) {
    if (info[b] != 0) throw std::runtime_error("dsyev failed. INFO=" + std::to_string(info[b]));
    const std::size_t dim = val[b].size(), keep = detail::nr_returned(DP, dim);
    out[b].val.assign(val[b].begin(), val[b].begin() + keep);
    if (keep == dim) {
      out[b].vec = std::move(vec[b]);
    } else {
      out[b].vec = M(keep, dim);
      for (std::size_t r = 0; r < keep; r++)
        for (std::size_t c = 0; c < dim; c++) out[b].vec(r, c) = vec[b](r, c);
    }
  }
  return out;
}

// diagonalise() of one block (c++/diag.hpp:261): m is read, not destroyed.
template <class M>
RawEigen<M> diagonalise(M& m, const DiagParams& DP = DiagParams(), int myrank = 0) {
  (void)myrank;
  std::vector<M> one;
  one.push_back(m);
  return std::move(diagonalisations(one, DP)[0]);
}

namespace detail {

template <class M, class A, class O, class B>
void gemm3(M& Mm, double factor, const A& Am, bool transA, const O* Om, const B& Bm) {
  // finite_size checks of the reference: a term with an empty factor contributes nothing
  const std::size_t rows = Mm.size1(), cols = Mm.size2();
  const std::size_t ka = transA ? Am.size1() : Am.size2();
  if (!Am.size1() || !Am.size2() || !Bm.size1() || !Bm.size2()) return;
  const std::size_t kb = Om ? Om->size2() : ka;
  const bool ok = (transA ? Am.size2() : Am.size1()) == rows && Bm.size2() == kb && Bm.size1() == cols &&
                  (!Om || Om->size1() == ka);
  if (!ok) throw std::invalid_argument("matrix shapes do not conform");
  nrg_gemm3 t{};
  t.M = base(Mm);
  t.ldm = static_cast<int64_t>(cols);
  t.A = base(Am);
  t.lda = static_cast<int64_t>(Am.size2());
  t.O = Om ? base(*Om) : nullptr;
  t.ldo = Om ? static_cast<int64_t>(Om->size2()) : 0;
  t.B = base(Bm);
  t.ldb = static_cast<int64_t>(Bm.size2());
  t.rows = static_cast<int>(rows);
  t.cols = static_cast<int>(cols);
  t.ka = static_cast<int>(ka);
  t.kb = static_cast<int>(kb);
  t.transA = transA ? 1 : 0;
  t.transB = 1;
  t.factor = factor;
  check(nrg_gemm3_batch_host(context(current_device()), 1, &t, nullptr), "nrg_gemm3_batch_host");
}

}  // namespace detail

// M += factor * A * B^T  (c++/numerics_ublas.hpp:108-116)
template <class M, class A, class B>
void product(M& Mm, double factor, const A& Am, const B& Bm) {
  detail::gemm3<M, A, A, B>(Mm, factor, Am, false, nullptr, Bm);
}

// M += factor * A * O * B^T  (c++/numerics_ublas.hpp:119-128; O * B^T is formed first)
template <class M, class A, class O, class B>
void transform(M& Mm, double factor, const A& Am, const O& Om, const B& Bm) {
  detail::gemm3(Mm, factor, Am, false, &Om, Bm);
}

// M += factor * U^T * O * U  (c++/numerics_ublas.hpp:130-140)
template <class M, class U, class O>
void rotate(M& Mm, double factor, const U& Um, const O& Om) {
  if (!Um.size1() || !Um.size2()) return;
  // U is n x dim: op(A) = U^T (dim x n), O is n x n, op(B) = U (B stored dim x n would be
  // U^T); the batched form takes B = U with transB = 0, so it is staged as such.
  const std::size_t rows = Mm.size1(), cols = Mm.size2(), n = Um.size1();
  if (Um.size2() != rows || Om.size1() != n || Om.size2() != n || cols != rows)
    throw std::invalid_argument("matrix shapes do not conform");
  nrg_gemm3 t{};
  t.M = detail::base(Mm);
  t.ldm = static_cast<int64_t>(cols);
  t.A = detail::base(Um);
  t.lda = static_cast<int64_t>(Um.size2());
  t.O = detail::base(Om);
  t.ldo = static_cast<int64_t>(Om.size2());
  t.B = detail::base(Um);
  t.ldb = static_cast<int64_t>(Um.size2());
  t.rows = static_cast<int>(rows);
  t.cols = static_cast<int>(cols);
  t.ka = static_cast<int>(n);
  t.kb = static_cast<int>(n);
  t.transA = 1;
  t.transB = 0;
  t.factor = factor;
  check(nrg_gemm3_batch_host(detail::context(current_device()), 1, &t, nullptr), "nrg_gemm3_batch_host");
}

}  // namespace nrg_b200

#endif  // NRG_B200_HPP
