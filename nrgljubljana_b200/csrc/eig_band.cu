// eig_band.cu -- two-stage reduction of the largest symmetric blocks to tridiagonal form,
// and the back-transform of its second stage.
//
// Replaces, for blocks above the band threshold of nrg_tuning, the one-stage Householder
// reduction that LAPACK dsyev/dsyevd perform inside diagonalise() (c++/diag.hpp:62-115 of
// the reference). The one-stage reduction streams the trailing matrix once per column
// (one FLOP per byte); for a few very large blocks its per-column chain bounds the step.
// Here:
//   stage 1  dense -> band of width kBand: per panel of kBand columns a Householder QR of
//            the panel (band_panel_kernel) and the two-sided update of the trailing matrix as
//            FP64 tensor-core GEMMs in compact-WY form (planned by eig_large.cu);
//   stage 2  band -> tridiagonal by bulge chasing (band_chase_kernel): one Householder
//            reflector of length kBand per step, sweeps pipelined over the warps of a CTA;
//   back     the reflectors of stage 2, grouped kGrp sweeps at a time into compact-WY
//            blocks (band_q2_tfactor_kernel), applied to the eigenvector rows
//            (band_q2_apply_kernel); stage 1's reflectors are left in the form of the
//            one-stage back-transform (row k: unit at k + kBand) and applied by it.
// Published methods: Householder reflectors as dlarfg (v0 = 1), the compact-WY
// representation (Schreiber-Van Loan), two-stage tridiagonalisation with bulge chasing
// (Bischof-Lang-Sun successive band reduction; pipelined sweeps as in Haidar-Ltaief-Dongarra).
#include <cuda_runtime.h>

#include "band.h"
#include "common.cuh"

namespace nrg {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBtPanel = 128;  // panel width of the one-stage back-transform (eig_large.cu)

// ---------------------------------------------------------------- stage 0: full symmetric copy
// S (n x lds, row-major) = the symmetric matrix whose upper triangle is H's (row-major).
// Grid (tiles of 32 x 32 over the largest block, blocks); 32 x 8 threads.
__global__ void __launch_bounds__(256) band_sym_kernel(const BandBlock* __restrict__ blocks) {
  const BandBlock B = blocks[blockIdx.y];
  const int n = B.n, nt = (n + 31) / 32;
  if ((int)blockIdx.x >= nt * nt) return;
  const int tr = blockIdx.x / nt, tc = blockIdx.x % nt;
  __shared__ double tile[32][33];
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
  const int sr = min(tr, tc), sc = max(tr, tc);  // the tile of H's upper triangle that holds it
  for (int r = ly; r < 32; r += 8) {
    const int gr = sr * 32 + r, gc = sc * 32 + lx;
    tile[r][lx] = (gr < n && gc < n) ? B.H[(size_t)gr * n + gc] : 0.0;
  }
  __syncthreads();
  for (int r = ly; r < 32; r += 8) {
    const int gr = tr * 32 + r, gc = tc * 32 + lx;
    if (gr >= n || gc >= n) continue;
    double v;
    if (tr < tc) v = tile[r][lx];
    else if (tr > tc) v = tile[lx][r];
    else v = (r <= lx) ? tile[r][lx] : tile[lx][r];
    B.S[(size_t)gr * B.lds + gc] = v;
  }
}

// ---------------------------------------------------------------- stage 1: panel QR
// Panel at column j0 of every block with m = n - j0 - kBand > 1 rows below the band. The
// panel's columns are held transposed in rows j0 .. j0+kBand-1 of the symmetric S:
// P(q, i) = S[(j0+q)*lds + j0 + kBand + i], i < m. On exit:
//   - BND holds the lower triangle of the diagonal block (rows/columns j0..j0+kBand-1) and
//     R, the panel's triangular factor (the band below the diagonal block);
//   - row k = j0+q of S holds reflector k in the back-transform's form: zeros from the start
//     of its back-transform panel up to k+kBand, 1 at k+kBand, v beyond -- which is also
//     exactly the kb x m matrix Vt that the GEMMs of the trailing update read;
//   - tau1[k], and T1 (kBand x kBand, zero-padded) of H_j0 ... H_j0+kb-1 = I - V T1 V^T.
__global__ void __launch_bounds__(256) band_panel_kernel(const BandBlock* __restrict__ blocks, int j0) {
  const BandBlock B = blocks[blockIdx.x];
  const int n = B.n, ld = B.lds, b = kBand;
  const int m = n - j0 - b;
  if (m <= 1) return;
  const int kb = min(b, m - 1);
  double* P = B.S + (size_t)j0 * ld + j0 + b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5, nt = blockDim.x;
  __shared__ double red[64];
  __shared__ double stau[kBand];
  __shared__ double G[kBand][kBand + 1];
  __shared__ double T[kBand][kBand + 1];
  __shared__ double wv[kBand];

  // 1. lower triangle of the diagonal block into the band
  for (int idx = tid; idx < b * b; idx += nt) {
    const int rr = idx / b, cc = idx % b;
    if (rr >= cc && j0 + rr < n) B.BND[(size_t)(j0 + cc) * kLDB + (rr - cc)] = B.S[(size_t)(j0 + rr) * ld + j0 + cc];
  }
  // 2. Householder QR, column by column; rows r > q (columns not yet factored) are owned by
  //    one warp each for the update
  for (int q = 0; q < kb; q++) {
    double* pq = P + (size_t)q * ld;
    double part = 0.0;
    for (int i = q + 1 + tid; i < m; i += nt) {
      const double x = pq[i];
      part += x * x;
    }
    const double sigma = block_sum(part, red);
    const double alpha = pq[q];
    double tau = 0.0, beta = alpha;
    if (sigma > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
      tau = (beta - alpha) / beta;
      const double scale = 1.0 / (alpha - beta);
      for (int i = q + 1 + tid; i < m; i += nt) pq[i] *= scale;
    }
    if (tid == 0) stau[q] = tau;
    __syncthreads();  // v_q complete; every thread has read alpha
    if (tau != 0.0) {
      for (int r = q + 1 + warp; r < b; r += nw) {
        double* pr = P + (size_t)r * ld;
        double s = 0.0;
        for (int i = q + 1 + lane; i < m; i += 32) s += pr[i] * pq[i];
        s = warp_sum(s) + pr[q];
        const double f = tau * s;
        __syncwarp();
        if (lane == 0) pr[q] -= f;
        for (int i = q + 1 + lane; i < m; i += 32) pr[i] -= f * pq[i];
      }
    }
    __syncthreads();
    if (tid == 0) pq[q] = beta;
    __syncthreads();
  }
  for (int q = kb + tid; q < b; q += nt) stau[q] = 0.0;
  __syncthreads();
  // 3. R into the band: A(j0+b+i, j0+q) = R(i, q) = P(q, i) for i <= q
  for (int idx = tid; idx < b * b; idx += nt) {
    const int q = idx / b, i = idx % b;
    if (i <= q && i < m && j0 + q < n) B.BND[(size_t)(j0 + q) * kLDB + (b + i - q)] = P[(size_t)q * ld + i];
  }
  // 4. Gram matrix G(q, r) = v_q . v_r for r < q < kb (v_r(q) = P(r, q)), then T1
  const int npair = kb * (kb - 1) / 2;
  for (int p = warp; p < npair; p += nw) {
    int q = 1;
    while ((q * (q + 1)) / 2 <= p) q++;
    const int r = p - (q * (q - 1)) / 2;
    const double* pq = P + (size_t)q * ld;
    const double* pr = P + (size_t)r * ld;
    double s = 0.0;
    for (int i = q + 1 + lane; i < m; i += 32) s += pq[i] * pr[i];
    s = warp_sum(s);
    if (lane == 0) G[q][r] = s + pr[q];
  }
  for (int idx = tid; idx < b * (b + 1); idx += nt) T[idx / (b + 1)][idx % (b + 1)] = 0.0;
  __syncthreads();
  for (int q = 0; q < kb; q++) {
    // T(0:q, q) = -tau_q T(0:q, 0:q) G(q, 0:q)^T
    if (tid < q) wv[tid] = -stau[q] * G[q][tid];
    __syncthreads();
    if (tid < q) {
      double s = 0.0;
      for (int r = tid; r < q; r++) s += T[tid][r] * wv[r];
      T[tid][q] = s;
    }
    if (tid == q) T[q][q] = stau[q];
    __syncthreads();
  }
  double* T1 = B.scr + band_scr_t(n);
  for (int idx = tid; idx < b * b; idx += nt) T1[idx] = T[idx / b][idx % b];
  for (int q = tid; q < b; q += nt)
    if (j0 + q < n) B.tau1[j0 + q] = stau[q];
  // 5. the rows in back-transform form: zeros from the reflector's back-transform panel start
  //    (+ kBand) up to k + kBand, the unit at k + kBand
  for (int q = 0; q < b; q++) {
    const int k = j0 + q;
    if (k >= n) break;
    double* row = B.S + (size_t)k * ld;
    const int c0 = (k / kBtPanel) * kBtPanel + b, c1 = min(k + b, n);
    for (int c = c0 + tid; c < c1; c += nt) row[c] = 0.0;
    if (tid == 0 && k + b < n) row[k + b] = 1.0;
  }
}

// ---------------------------------------------------------------- stage 2: bulge chasing
// Lower band storage: A(c + t, c) at BND[c*kLDB + t], t <= 2 kBand. Step j of sweep i
// builds the reflector that clears column col (col = i for j = 0, else the first column of
// the previous step's rows) below row r0 = i+1+j*kBand over the rows r0 .. r0+L-1, and
// applies it where the band holds nonzeros: from the left to the columns col+1 .. r0-1 of
// those rows (the rest of the previous bulge), from both sides to the diagonal block, from
// the right to the kBand rows below (the new bulge). The fill never passes distance
// 2 kBand - 1 from the diagonal. Lane t owns row r0+t. Band loads bypass L1 (ld.global.cg):
// other warps of the CTA wrote them.
NRG_DEV double bld(const double* band, int c, int t) { return __ldcg(band + (size_t)c * kLDB + t); }
NRG_DEV void bst(double* band, int c, int t, double x) { band[(size_t)c * kLDB + t] = x; }

NRG_DEV void chase_step(double* __restrict__ band, double* __restrict__ V2, double* __restrict__ tau2, int n,
                        int J, int i, int j, int lane, double* vs, double* ws) {
  const int r0 = i + 1 + j * kBand, L = min(kBand, n - r0);
  const int col = j == 0 ? i : r0 - kBand;
  const double x = lane < L ? bld(band, col, r0 + lane - col) : 0.0;
  const double sigma = warp_sum((lane >= 1 && lane < L) ? x * x : 0.0);
  const double alpha = __shfl_sync(kFull, x, 0);
  double tau = 0.0, beta = alpha, v = lane == 0 ? 1.0 : 0.0;
  if (sigma > 0.0) {
    beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
    tau = (beta - alpha) / beta;
    if (lane >= 1 && lane < L) v = x / (alpha - beta);
  }
  const size_t ro = (size_t)i * J + j;
  V2[ro * kBand + lane] = v;  // zero beyond L
  if (lane == 0) tau2[ro] = tau;
  if (lane < L) bst(band, col, r0 + lane - col, lane == 0 ? beta : 0.0);
  if (tau == 0.0) return;
  vs[lane] = v;
  __syncwarp();
  // Each phase first loads its operands into registers (all loads in flight at once), then
  // computes and stores.
  double a[kBand];
  // left: the previous bulge's other columns col+1 .. r0-1 (nl <= kBand - 1 of them)
  const int nl = r0 - col - 1;
#pragma unroll
  for (int cc = 0; cc < kBand - 1; cc++)
    a[cc] = (cc < nl && lane < L) ? bld(band, col + 1 + cc, r0 + lane - col - 1 - cc) : 0.0;
#pragma unroll
  for (int cc = 0; cc < kBand - 1; cc++) {
    if (cc < nl) {
      const double w = warp_sum(v * a[cc]);
      if (lane < L) bst(band, col + 1 + cc, r0 + lane - col - 1 - cc, a[cc] - tau * v * w);
    }
  }
  // both sides: the diagonal block D (L x L, symmetric, lower part stored); lane t holds row t
#pragma unroll
  for (int s = 0; s < kBand; s++)
    a[s] = (lane < L && s < L) ? (s <= lane ? bld(band, r0 + s, lane - s) : bld(band, r0 + lane, s - lane)) : 0.0;
  double p = 0.0;
#pragma unroll
  for (int s = 0; s < kBand; s++) p += a[s] * vs[s];
  p *= tau;
  const double K = 0.5 * tau * warp_sum(p * v);
  const double w = p - K * v;
  ws[lane] = w;
  __syncwarp();
#pragma unroll
  for (int s = 0; s < kBand; s++)
    if (lane < L && s <= lane) bst(band, r0 + s, lane - s, a[s] - (v * ws[s] + w * vs[s]));
  // right: the kBand rows below the block (the new bulge); lane u holds row r1+u
  const int r1 = r0 + L, L2 = min(kBand, n - r1);
  if (L2 > 0) {
#pragma unroll
    for (int s = 0; s < kBand; s++) a[s] = (lane < L2 && s < L) ? bld(band, r0 + s, r1 + lane - r0 - s) : 0.0;
    double y = 0.0;
#pragma unroll
    for (int s = 0; s < kBand; s++) y += a[s] * vs[s];
    y *= tau;
#pragma unroll
    for (int s = 0; s < kBand; s++)
      if (lane < L2 && s < L) bst(band, r0 + s, r1 + lane - r0 - s, a[s] - y * vs[s]);
  }
  __syncwarp();
}

// One CTA per block; warp w runs sweeps w, w + kChaseWarps, ... Step j of sweep i waits until
// sweep i-1 has finished step j+3 (from step j+4 on, the two sweeps touch disjoint index
// ranges). Progress per warp: key(i, c) = i*(J+1) + c after c steps of sweep i (c = J when
// the sweep is done), monotone. Waits are bounded: if one runs out the CTA stops and marks
// the block's status word.
__global__ void __launch_bounds__(32 * kChaseWarps) band_chase_kernel(const BandBlock* __restrict__ blocks) {
  const BandBlock B = blocks[blockIdx.x];
  const int n = B.n, J = B.J, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ volatile int prog[kChaseWarps];
  __shared__ volatile int abort_flag;
  __shared__ double vsh[kChaseWarps][kBand], wsh[kChaseWarps][kBand];
  // the final diagonal block [jfin, n) of S into the band (its distances <= kBand)
  for (int idx = tid; idx < (n - B.jfin) * (kBand + 1); idx += blockDim.x) {
    const int c = B.jfin + idx / (kBand + 1), t = idx % (kBand + 1);
    if (c + t < n) B.BND[(size_t)c * kLDB + t] = B.S[(size_t)(c + t) * B.lds + c];
  }
  if (tid < kChaseWarps) prog[tid] = -1;
  if (tid == 0) abort_flag = 0;
  __threadfence_block();
  __syncthreads();
  const int nsw = band_nsweeps(n);
  bool stop = false;  // warp-uniform
  for (int i = warp; i < nsw && !stop; i += kChaseWarps) {
    const int ns = band_nsteps(n, i);
    for (int j = 0; j < ns; j++) {
      if (i > 0) {
        const int wp = (i - 1) % kChaseWarps;
        const int need = (i - 1) * (J + 1) + min(j + 4, J);
        int ok = 1;
        if (lane == 0) {
          long long it = 0;
          while (prog[wp] < need) {
            if (abort_flag) break;
            if (++it > (1LL << 24)) {
              abort_flag = 1;
              break;
            }
            __nanosleep(64);
          }
          ok = prog[wp] >= need;
        }
        ok = __shfl_sync(kFull, ok, 0);
        if (!ok) {
          stop = true;
          break;
        }
        __threadfence_block();
      }
      chase_step(B.BND, B.V2, B.tau2, n, J, i, j, lane, vsh[warp], wsh[warp]);
      __syncwarp();
      __threadfence_block();
      if (lane == 0) prog[warp] = i * (J + 1) + (j + 1 == ns ? J : j + 1);
    }
  }
  __syncthreads();
  if (abort_flag) {
    if (tid == 0) *B.info = 1;  // the chase did not finish: not converged, no result
    return;
  }
  for (int c = tid; c < n; c += blockDim.x) {
    B.d[c] = bld(B.BND, c, 0);
    B.e[c] = c + 1 < n ? bld(B.BND, c, 1) : 0.0;
  }
}

// ---------------------------------------------------------------- stage 2 back-transform
// Group (g, j): the reflectors of step j of sweeps g*kGrp .. g*kGrp + kGrp - 1 (those that
// have a step j, a prefix). Member q acts on rows rs + q .. rs + q + kBand - 1 with
// rs = g*kGrp + 1 + j*kBand, so the group's matrix V (rows rs .., columns q) is a
// parallelogram of kBand + kGrp - 1 rows. Their product in sweep order is I - V T V^T.
NRG_DEV int group_members(int n, int g, int j) {
  const int i0 = g * kGrp;
  int q = 0;
  while (q < kGrp && i0 + q < band_nsweeps(n) && band_nsteps(n, i0 + q) > j) q++;
  return q;
}

constexpr int kGRows = kBand + kGrp - 1;  // rows of a group's V

// Grid (groups g*J + j of the largest block, blocks); 128 threads.
__global__ void __launch_bounds__(128) band_q2_tfactor_kernel(const BandBlock* __restrict__ blocks) {
  const BandBlock B = blocks[blockIdx.y];
  const int n = B.n, J = B.J;
  const int g = blockIdx.x / max(J, 1), j = blockIdx.x % max(J, 1);
  if (J == 0 || g >= band_ngroups(n)) return;
  const int nm = group_members(n, g, j);
  if (nm == 0) return;
  __shared__ double V[kGrp][kGRows + 1];
  __shared__ double Gm[kGrp][kGrp + 1];
  __shared__ double T[kGrp][kGrp + 1];
  __shared__ double tv[kGrp], wv[kGrp];
  const int tid = threadIdx.x;
  for (int idx = tid; idx < kGrp * kGRows; idx += blockDim.x) {
    const int q = idx / kGRows, r = idx % kGRows;
    double x = 0.0;
    if (q < nm && r >= q && r < q + kBand) x = B.V2[((size_t)(g * kGrp + q) * J + j) * kBand + (r - q)];
    V[q][r] = x;
  }
  if (tid < kGrp) tv[tid] = tid < nm ? B.tau2[(size_t)(g * kGrp + tid) * J + j] : 0.0;
  __syncthreads();
  for (int idx = tid; idx < kGrp * kGrp; idx += blockDim.x) {
    const int q = idx / kGrp, r = idx % kGrp;
    double s = 0.0;
    if (r < q)
      for (int k = q; k < r + kBand; k++) s += V[q][k] * V[r][k];
    Gm[q][r] = s;
    T[q][r] = 0.0;
  }
  __syncthreads();
  for (int q = 0; q < nm; q++) {
    if (tid < q) wv[tid] = -tv[q] * Gm[q][tid];
    __syncthreads();
    if (tid < q) {
      double s = 0.0;
      for (int r = tid; r < q; r++) s += T[tid][r] * wv[r];
      T[tid][q] = s;
    }
    if (tid == q) T[q][q] = tv[q];
    __syncthreads();
  }
  double* out = B.T2 + ((size_t)g * J + j) * kGrp * kGrp;
  for (int idx = tid; idx < kGrp * kGrp; idx += blockDim.x) out[idx] = T[idx / kGrp][idx % kGrp];
}

// The eigenvector rows Zt (evecs, n x n) times Q2^T: for every group, in the order of the
// product (groups g descending, steps j ascending), Zt[:, R] -= ((Zt[:, R] V) T^T) V^T.
// Each CTA owns kQ2Rows eigenvector rows and walks all groups. Per group the three small
// products run on the FP64 tensor cores (DMMA m8n8k4) from shared memory, zero-padded to
// 64 x 64 (window), 32 x 64 (V) and 32 x 32 (T); 8 warps.
constexpr int kQ2Rows = 64;
static_assert(kGRows <= 64 && kGrp == 32 && kQ2Rows == 64, "the DMMA tiling below assumes these shapes");
constexpr int kLW = 68;  // row stride (doubles) of the window and of V in shared memory
constexpr int kLX = 36;  // row stride of X, X2 and T

__global__ void __launch_bounds__(256) band_q2_apply_kernel(const BandBlock* __restrict__ blocks) {
  const BandBlock B = blocks[blockIdx.y];
  const int n = B.n, J = B.J;
  const int e0 = blockIdx.x * kQ2Rows;
  if (e0 >= n || J == 0) return;
  const int ne = min(kQ2Rows, n - e0);
  extern __shared__ __align__(16) double q2sm[];
  double* W = q2sm;                  // 64 x kLW: the window Zt[e0 .., R]
  double* V = W + 64 * kLW;          // 32 x kLW: row q = reflector q over the window's columns
  double* T = V + 32 * kLW;          // 32 x kLX
  double* X = T + 32 * kLX;          // 64 x kLX
  double* X2 = X + 64 * kLX;         // 64 x kLX
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int fr = lane >> 2, fc = lane & 3;
  for (int g = band_ngroups(n) - 1; g >= 0; g--) {
    for (int j = 0; j < J; j++) {
      const int nm = group_members(n, g, j);
      if (nm == 0) break;  // members form a prefix in j as well: no later step has any
      const int rs = g * kGrp + 1 + j * kBand;
      const int nr = min(kGRows, n - rs);
      for (int idx = tid; idx < 32 * 64; idx += nt) {
        const int q = idx >> 6, r = idx & 63;
        double x = 0.0;
        if (q < nm && r >= q && r < q + kBand && r < nr)
          x = B.V2[((size_t)(g * kGrp + q) * J + j) * kBand + (r - q)];
        V[q * kLW + r] = x;
      }
      const double* Tg = B.T2 + ((size_t)g * J + j) * kGrp * kGrp;
      for (int idx = tid; idx < kGrp * kGrp; idx += nt) T[(idx / kGrp) * kLX + idx % kGrp] = Tg[idx];
      for (int idx = tid; idx < 64 * 64; idx += nt) {
        const int e = idx >> 6, r = idx & 63;
        W[e * kLW + r] = (e < ne && r < nr) ? B.evecs[(size_t)(e0 + e) * n + rs + r] : 0.0;
      }
      __syncthreads();
      const int rb = (warp >> 1) * 16;  // the warp's 16 rows
      // X (64 x 32) = W V^T, K = 64: warp tile 16 x 16
      {
        const int cb = (warp & 1) * 16;
        double acc[2][2][2] = {};
        for (int k0 = 0; k0 < 64; k0 += 4) {
          double a[2], bb[2];
#pragma unroll
          for (int i = 0; i < 2; i++) a[i] = W[(rb + 8 * i + fr) * kLW + k0 + fc];
#pragma unroll
          for (int jj = 0; jj < 2; jj++) bb[jj] = V[(cb + 8 * jj + fr) * kLW + k0 + fc];
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int jj = 0; jj < 2; jj++) dmma884(acc[i][jj][0], acc[i][jj][1], a[i], bb[jj]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int h = 0; h < 2; h++) X[(rb + 8 * i + fr) * kLX + cb + 8 * jj + 2 * fc + h] = acc[i][jj][h];
      }
      __syncthreads();
      // X2 (64 x 32) = X T^T, K = 32
      {
        const int cb = (warp & 1) * 16;
        double acc[2][2][2] = {};
        for (int k0 = 0; k0 < 32; k0 += 4) {
          double a[2], bb[2];
#pragma unroll
          for (int i = 0; i < 2; i++) a[i] = X[(rb + 8 * i + fr) * kLX + k0 + fc];
#pragma unroll
          for (int jj = 0; jj < 2; jj++) bb[jj] = T[(cb + 8 * jj + fr) * kLX + k0 + fc];
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int jj = 0; jj < 2; jj++) dmma884(acc[i][jj][0], acc[i][jj][1], a[i], bb[jj]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int h = 0; h < 2; h++) X2[(rb + 8 * i + fr) * kLX + cb + 8 * jj + 2 * fc + h] = acc[i][jj][h];
      }
      __syncthreads();
      // W -= X2 V (64 x 64, K = 32): warp tile 16 x 32, written back to the eigenvector rows
      {
        const int cb = (warp & 1) * 32;
        double acc[2][4][2] = {};
        for (int k0 = 0; k0 < 32; k0 += 4) {
          double a[2], bb[4];
#pragma unroll
          for (int i = 0; i < 2; i++) a[i] = X2[(rb + 8 * i + fr) * kLX + k0 + fc];
#pragma unroll
          for (int jj = 0; jj < 4; jj++) bb[jj] = V[(k0 + fc) * kLW + cb + 8 * jj + fr];
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int jj = 0; jj < 4; jj++) dmma884(acc[i][jj][0], acc[i][jj][1], a[i], bb[jj]);
        }
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int e = rb + 8 * i + fr;
          if (e >= ne) continue;
#pragma unroll
          for (int jj = 0; jj < 4; jj++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const int r = cb + 8 * jj + 2 * fc + h;
              if (r < nr) B.evecs[(size_t)(e0 + e) * n + rs + r] = W[e * kLW + r] - acc[i][jj][h];
            }
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace

cudaError_t band_sym_launch(const BandBlock* d_blocks, int nblk, int maxn, cudaStream_t s) {
  if (nblk <= 0) return cudaSuccess;
  const int nt = (maxn + 31) / 32;
  band_sym_kernel<<<dim3((unsigned)(nt * nt), (unsigned)nblk), 256, 0, s>>>(d_blocks);
  return cudaGetLastError();
}

cudaError_t band_panel_launch(const BandBlock* d_blocks, int nactive, int j0, cudaStream_t s) {
  if (nactive <= 0) return cudaSuccess;
  band_panel_kernel<<<nactive, 256, 0, s>>>(d_blocks, j0);
  return cudaGetLastError();
}

cudaError_t band_chase_launch(const BandBlock* d_blocks, int nblk, cudaStream_t s) {
  if (nblk <= 0) return cudaSuccess;
  band_chase_kernel<<<nblk, 32 * kChaseWarps, 0, s>>>(d_blocks);
  return cudaGetLastError();
}

cudaError_t band_q2_tfactor_launch(const BandBlock* d_blocks, int nblk, int maxn, cudaStream_t s) {
  if (nblk <= 0) return cudaSuccess;
  const int J = band_nsteps(maxn, 0), G = band_ngroups(maxn);
  if (J == 0 || G == 0) return cudaSuccess;
  band_q2_tfactor_kernel<<<dim3((unsigned)(G * J), (unsigned)nblk), 128, 0, s>>>(d_blocks);
  return cudaGetLastError();
}

cudaError_t band_q2_apply_launch(const BandBlock* d_blocks, int nblk, int maxn, cudaStream_t s) {
  if (nblk <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * (64 * kLW + 32 * kLW + 32 * kLX + 2 * 64 * kLX);
  cudaError_t err = cudaFuncSetAttribute(band_q2_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  band_q2_apply_kernel<<<dim3((unsigned)((maxn + kQ2Rows - 1) / kQ2Rows), (unsigned)nblk), 256, smem, s>>>(d_blocks);
  return cudaGetLastError();
}

}  // namespace nrg
