// eig_small.cuh -- shared-memory building blocks of the one-CTA eigensolver:
// Householder tridiagonalisation of a dense symmetric matrix held in shared memory,
// explicit formation of the orthogonal factor, and the implicit-shift QL iteration on a
// symmetric tridiagonal matrix with rotation accumulation.
//
// Control flow is uniform across the CTA: one thread computes the serial rotation chain
// of a QL sweep into shared memory, every thread then applies it to its rows.
#pragma once
#include "common.cuh"

namespace nrg {

// Householder reduction A = Q T Q^T of the symmetric n x n matrix A (both triangles,
// row stride ld) in shared memory. On exit d[0..n) is the diagonal and e[0..n-1) the
// sub-diagonal of T (e[n-1] = 0); column k of A below the sub-diagonal holds the
// Householder vector v_k (v_k[k+1] = 1 stored explicitly) and taus[k] its scalar.
// Scratch: vw (2n doubles), red (32 doubles).
NRG_DEV void smem_tridiagonalise(double* A, int ld, int n, double* d, double* e, double* taus, double* vw,
                                 double* red) {
  const int tid = threadIdx.x, nt = blockDim.x;
  double* v = vw;
  double* w = vw + n;
  for (int k = 0; k + 2 < n; k++) {
    // sigma = sum of squares below the sub-diagonal entry of column k
    double part = 0.0;
    for (int i = k + 2 + tid; i < n; i += nt) {
      const double x = A[i * ld + k];
      part += x * x;
    }
    const double sigma = block_sum(part, red);
    const double alpha = A[(k + 1) * ld + k];
    double tau = 0.0, beta = alpha;
    if (sigma > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
      tau = (beta - alpha) / beta;
      const double scale = 1.0 / (alpha - beta);
      for (int i = k + 2 + tid; i < n; i += nt) v[i] = A[i * ld + k] * scale;
    } else {
      for (int i = k + 2 + tid; i < n; i += nt) v[i] = A[i * ld + k];
    }
    if (tid == 0) {
      v[k + 1] = 1.0;
      e[k] = beta;
      taus[k] = tau;
    }
    __syncthreads();
    if (tau != 0.0) {
      // w = tau * A22 * v over the trailing block [k+1, n)
      for (int i = k + 1 + tid; i < n; i += nt) {
        double s = 0.0;
        for (int j = k + 1; j < n; j++) s += A[i * ld + j] * v[j];
        w[i] = tau * s;
      }
      __syncthreads();
      double pp = 0.0;
      for (int i = k + 1 + tid; i < n; i += nt) pp += w[i] * v[i];
      const double K = 0.5 * tau * block_sum(pp, red);
      for (int i = k + 1 + tid; i < n; i += nt) w[i] -= K * v[i];
      __syncthreads();
      const int m = n - k - 1;
      for (int idx = tid; idx < m * m; idx += nt) {
        const int i = k + 1 + idx / m, j = k + 1 + idx % m;
        A[i * ld + j] -= v[i] * w[j] + w[i] * v[j];
      }
      __syncthreads();
    }
    // keep v_k in column k for the formation of Q
    for (int i = k + 1 + tid; i < n; i += nt) A[i * ld + k] = v[i];
    if (tid == 0) d[k] = A[k * ld + k];
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A[(n - 2) * ld + (n - 2)];
      e[n - 2] = A[(n - 1) * ld + (n - 2)];
      if (n >= 3) taus[n - 2] = 0.0;
    }
    d[n - 1] = A[(n - 1) * ld + (n - 1)];
    e[n - 1] = 0.0;
  }
  __syncthreads();
}

// Z = H_0 H_1 ... H_{n-3} from the vectors left in A by smem_tridiagonalise (backward
// accumulation). Z has row stride ld. Scratch s (n doubles).
NRG_DEV void smem_form_q(const double* A, int ld, int n, const double* taus, double* Z, double* s) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int idx = tid; idx < n * n; idx += nt) {
    const int i = idx / n, j = idx % n;
    Z[i * ld + j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int k = n - 3; k >= 0; k--) {
    const double tau = taus[k];
    if (tau == 0.0) continue;  // uniform: taus is shared
    for (int j = k + 1 + tid; j < n; j += nt) {
      double t = 0.0;
      for (int i = k + 1; i < n; i++) t += A[i * ld + k] * Z[i * ld + j];
      s[j] = tau * t;
    }
    __syncthreads();
    const int m = n - k - 1;
    for (int idx = tid; idx < m * m; idx += nt) {
      const int i = k + 1 + idx / m, j = k + 1 + idx % m;
      Z[i * ld + j] -= A[i * ld + k] * s[j];
    }
    __syncthreads();
  }
}

// sqrt(f^2 + g^2) with one square root while the squares can neither overflow nor lose
// their low bits to underflow; the scaled library hypot otherwise.
NRG_DEV double chain_hypot(double f, double g) {
  const double mx = fmax(fabs(f), fabs(g));
  if (mx > 1e-140 && mx < 1e140) return sqrt(fma(f, f, g * g));
  return hypot(f, g);
}

// Implicit-shift QL iteration (Wilkinson-type shift) on the symmetric tridiagonal matrix
// (d, e), e[i] coupling i and i+1, e[n-1] unused. Rotations are accumulated into the
// columns of Z (nz rows, row stride ld): on exit column r of Z is the eigenvector of d[r].
// Eigenvalues are not sorted. C, S: 2n doubles each of scratch (two buffers of rotations);
// ctl: 8 ints of scratch. Needs at least 64 threads.
// The sweeps are pipelined: thread 0 runs the convergence test and the rotation chain of
// sweep t+1 (a serial recurrence through d and e) while the threads of the other warps apply
// the rotations of sweep t to the rows of Z. Each row gets every sweep's rotations in the same
// order as without the overlap, so the results are the same.
// Returns 0, or l+1 if eigenvalue l failed to converge within 30 sweeps.
NRG_DEV int smem_ql(double* d, double* e, int n, double* Z, int ld, int nz, double* C, double* S, int* ctl) {
  const int tid = threadIdx.x, nt = blockDim.x;
  // thread 0's state: current eigenvalue l, sweeps spent on it, status
  int l = 0, iter = 0, status = 0;
  // Finds the next sweep and computes its rotations into buffer `buf` (thread 0 only);
  // returns false when every eigenvalue has converged or one failed to.
  auto next_sweep = [&](int buf) -> bool {
    double* Cb = C + (size_t)buf * n;
    double* Sb = S + (size_t)buf * n;
    while (l < n) {
      int m = l;
      while (m < n - 1) {
        const double dd = fabs(d[m]) + fabs(d[m + 1]);
        if (fabs(e[m]) <= kEps * dd) break;
        m++;
      }
      if (m == l) {
        l++;
        iter = 0;
        continue;
      }
      if (iter++ == 30) {
        status = l + 1;
        return false;
      }
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      int lo = l;
      bool under = false;
      for (int i = m - 1; i >= l; i--) {
        const double f = s * e[i], b = c * e[i];
        r = chain_hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          lo = i + 1;
          under = true;
          break;
        }
        const double ir = 1.0 / r;
        s = f * ir;
        c = g * ir;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        Cb[i] = c;
        Sb[i] = s;
      }
      if (!under) {
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
      ctl[2 * buf] = lo;
      ctl[2 * buf + 1] = m - 1;
      return true;
    }
    return false;
  };
  if (tid == 0) {
    e[n - 1] = 0.0;
    ctl[4] = next_sweep(0) ? 1 : 0;
  }
  __syncthreads();
  for (int buf = 0;; buf ^= 1) {
    const int has = ctl[4], lo = ctl[2 * buf], hi = ctl[2 * buf + 1];
    __syncthreads();  // every thread has read ctl before thread 0 rewrites it
    if (!has) break;
    if (tid == 0) {
      ctl[4] = next_sweep(buf ^ 1) ? 1 : 0;
    } else if (tid >= 32) {
      const double* Cb = C + (size_t)buf * n;
      const double* Sb = S + (size_t)buf * n;
      for (int row = tid - 32; row < nz; row += nt - 32) {
        double* z = Z + row * ld;
        for (int i = hi; i >= lo; i--) {
          const double f = z[i + 1];
          const double zi = z[i];
          z[i + 1] = Sb[i] * zi + Cb[i] * f;
          z[i] = Cb[i] * zi - Sb[i] * f;
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0) ctl[5] = status;
  __syncthreads();
  return ctl[5];
}

// Stable ascending order of d[0..n) into perm (single thread, small n).
NRG_DEV void serial_sort_perm(const double* d, int n, int* perm) {
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int i = 1; i < n; i++) {  // insertion sort
    const int pi = perm[i];
    const double di = d[pi];
    int j = i - 1;
    while (j >= 0 && d[perm[j]] > di) {
      perm[j + 1] = perm[j];
      j--;
    }
    perm[j + 1] = pi;
  }
}

}  // namespace nrg
