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
#include <cooperative_groups.h>
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
// P(q, i) = S[(j0+q)*lds + j0 + kBand + i], i < m. One thread-block cluster of PC CTAs per
// block: CTA r keeps P(:, i) for its share of i in shared memory; the Householder QR runs
// column by column, each column's norm and the dot products of the remaining panel rows with
// its reflector summed over the cluster through distributed shared memory (every CTA sums the
// shares in the same order, so all hold the same scalars): two cluster barriers per column.
// On exit:
//   - BND holds the lower triangle of the diagonal block (rows/columns j0..j0+kBand-1) and
//     R, the panel's triangular factor (the band below the diagonal block);
//   - row k = j0+q of S holds reflector k in the back-transform's form: zeros from the start
//     of its back-transform panel up to k+kBand, 1 at k+kBand, v beyond -- which is also
//     exactly the kb x m matrix Vt that the GEMMs of the trailing update read;
//   - tau1[k], and T1 (kBand x kBand, zero-padded) of H_j0 ... H_j0+kb-1 = I - V T1 V^T.
constexpr int kPanelThreads = 256;
constexpr int kPanelPairs = kBand * (kBand - 1) / 2;

__global__ void __launch_bounds__(kPanelThreads) band_panel_kernel(const BandBlock* __restrict__ blocks, int j0,
                                                                   int chunk_max) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int PC = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const BandBlock B = blocks[blockIdx.x / PC];
  const int n = B.n, ld = B.lds, b = kBand;
  const int m = n - j0 - b;
  const bool active = m > 1;  // every CTA of the cluster takes every barrier either way
  const int kb = active ? min(b, m - 1) : 0;
  const int chunk = active ? (m + PC - 1) / PC : 0;
  const int c0 = active ? min(m, rank * chunk) : 0, c1 = active ? min(m, c0 + chunk) : 0, nc = c1 - c0;
  double* P = B.S + (size_t)j0 * ld + j0 + b;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = kPanelThreads / 32;
  extern __shared__ __align__(16) double psm[];
  const int lp = chunk_max + 1;              // row stride of the slab
  double* Ps = psm;                          // kBand x lp: P(q, c0 + i)
  double* sig = Ps + (size_t)b * lp;         // 2: this CTA's share of sigma, and alpha if it owns column q
  double* dots = sig + 2;                    // kBand: shares of the dot products
  double* gram = dots + b;                   // kPanelPairs: shares of the Gram matrix
  double* red = gram + kPanelPairs;          // 64
  __shared__ double Tsm[kBand][kBand + 1];
  __shared__ double wv[kBand], stau[kBand];

  for (int idx = tid; idx < b * nc; idx += kPanelThreads) {
    const int q = idx / nc, i = idx % nc;
    Ps[q * lp + i] = P[(size_t)q * ld + c0 + i];
  }
  if (rank == 0 && active)  // lower triangle of the diagonal block into the band
    for (int idx = tid; idx < b * b; idx += kPanelThreads) {
      const int rr = idx / b, cc = idx % b;
      if (rr >= cc && j0 + rr < n)
        B.BND[(size_t)(j0 + cc) * kLDB + (rr - cc)] = B.S[(size_t)(j0 + rr) * ld + j0 + cc];
    }
  __syncthreads();
  for (int q = 0; q < kb; q++) {
    double* pq = Ps + (size_t)q * lp;
    // this CTA's share of sigma = sum_{i > q} P(q, i)^2; alpha = P(q, q) from its owner
    double part = 0.0;
    for (int i = max(q + 1 - c0, 0) + tid; i < nc; i += kPanelThreads) part += pq[i] * pq[i];
    part = block_sum(part, red);
    if (tid == 0) {
      sig[0] = part;
      sig[1] = (q >= c0 && q < c1) ? pq[q - c0] : 0.0;
    }
    cl.sync();  // (1) shares of sigma and alpha
    double sigma = 0.0, alpha = 0.0;
    for (int r = 0; r < PC; r++) {
      const double* rs = cl.map_shared_rank(sig, r);
      sigma += rs[0];
      alpha += rs[1];
    }
    double tau = 0.0, beta = alpha, scale = 1.0;
    if (sigma > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
      tau = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
      for (int i = max(q + 1 - c0, 0) + tid; i < nc; i += kPanelThreads) pq[i] *= scale;
    }
    if (tid == 0) stau[q] = tau;
    __syncthreads();
    // shares of w_r = v . P(r, :) for r > q (v(q) = 1, v(i > q) = the scaled row q)
    for (int r = q + 1 + warp; r < b; r += nw) {
      const double* pr = Ps + (size_t)r * lp;
      double s = 0.0;
      for (int i = max(q - c0, 0) + lane; i < nc; i += 32) s += pr[i] * (i + c0 == q ? 1.0 : pq[i]);
      s = warp_sum(s);
      if (lane == 0) dots[r] = s;
    }
    cl.sync();  // (2) shares of the dot products
    if (tau != 0.0) {
      for (int r = q + 1 + warp; r < b; r += nw) {
        double w = 0.0;
        for (int k = 0; k < PC; k++) w += cl.map_shared_rank(dots, k)[r];
        const double f = tau * w;
        double* pr = Ps + (size_t)r * lp;
        for (int i = max(q - c0, 0) + lane; i < nc; i += 32) pr[i] -= f * (i + c0 == q ? 1.0 : pq[i]);
      }
    }
    if (tid == 0 && q >= c0 && q < c1) pq[q - c0] = beta;
    __syncthreads();
  }
  for (int q = kb + tid; q < b; q += kPanelThreads) stau[q] = 0.0;
  // shares of the Gram matrix G(q, r) = v_q . v_r, r < q < kb
  for (int p = warp; p < kPanelPairs; p += nw) {
    int q = 1;
    while ((q * (q + 1)) / 2 <= p) q++;
    const int r = p - (q * (q - 1)) / 2;
    double s = 0.0;
    if (q < kb) {
      const double* pq = Ps + (size_t)q * lp;
      const double* pr = Ps + (size_t)r * lp;
      for (int i = max(q - c0, 0) + lane; i < nc; i += 32) s += (i + c0 == q ? 1.0 : pq[i]) * pr[i];
    }
    s = warp_sum(s);
    if (lane == 0) gram[p] = s;
  }
  __syncthreads();
  // the panel rows back in back-transform form (zeros up to the unit), and R into the band
  for (int idx = tid; idx < b * nc; idx += kPanelThreads) {
    const int q = idx / nc, i = idx % nc, gi = c0 + i;
    const double x = Ps[q * lp + i];
    if (gi <= q && q < b && j0 + q < n) B.BND[(size_t)(j0 + q) * kLDB + (b + gi - q)] = x;  // R(gi, q)
    P[(size_t)q * ld + gi] = gi < q ? 0.0 : (gi == q ? 1.0 : x);
  }
  cl.sync();  // (3) every share of the Gram matrix is complete
  if (rank == 0 && active) {
    // zeros left of the panel from the reflector's back-transform panel start (+ kBand)
    for (int q = 0; q < b; q++) {
      const int k = j0 + q;
      if (k >= n) break;
      double* row = B.S + (size_t)k * ld;
      const int cz0 = (k / kBtPanel) * kBtPanel + b, cz1 = min(j0 + b, n);
      for (int c = cz0 + tid; c < cz1; c += kPanelThreads) row[c] = 0.0;
    }
    // T1 from the summed Gram matrix
    for (int idx = tid; idx < b * (b + 1); idx += kPanelThreads) Tsm[idx / (b + 1)][idx % (b + 1)] = 0.0;
    __syncthreads();
    for (int q = 0; q < kb; q++) {
      if (tid < q) {
        const int p = (q * (q - 1)) / 2 + tid;
        double g = 0.0;
        for (int k = 0; k < PC; k++) g += cl.map_shared_rank(gram, k)[p];
        wv[tid] = -stau[q] * g;
      }
      __syncthreads();
      if (tid < q) {
        double s = 0.0;
        for (int r = tid; r < q; r++) s += Tsm[tid][r] * wv[r];
        Tsm[tid][q] = s;
      }
      if (tid == q) Tsm[q][q] = stau[q];
      __syncthreads();
    }
    double* T1 = B.scr + band_scr_t(n);
    for (int idx = tid; idx < b * b; idx += kPanelThreads) T1[idx] = Tsm[idx / b][idx % b];
    for (int q = tid; q < b; q += kPanelThreads)
      if (j0 + q < n) B.tau1[j0 + q] = stau[q];
  }
  cl.sync();  // (4) no CTA leaves while another may still read its shared memory
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
                        int J, int i, int j, int lane, double* vs, double* ws, double* lt) {
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
  if (nl > 0) {
#pragma unroll
    for (int cc = 0; cc < kBand - 1; cc++)
      a[cc] = (cc < nl && lane < L) ? bld(band, col + 1 + cc, r0 + lane - col - 1 - cc) : 0.0;
    // w_c = sum_t v_t A(r0+t, c) by lane c, through a transpose in shared memory (lt: 32 x 33)
#pragma unroll
    for (int cc = 0; cc < kBand - 1; cc++) lt[lane * (kBand + 1) + cc] = a[cc];
    __syncwarp();
    double wc = 0.0;
    if (lane < nl)
      for (int t = 0; t < L; t++) wc += vs[t] * lt[t * (kBand + 1) + lane];
    ws[lane] = wc;
    __syncwarp();
#pragma unroll
    for (int cc = 0; cc < kBand - 1; cc++)
      if (cc < nl && lane < L) bst(band, col + 1 + cc, r0 + lane - col - 1 - cc, a[cc] - tau * v * ws[cc]);
    __syncwarp();  // ws is rewritten below
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

// Orders this thread's memory accesses at cluster scope: the band is read and written only by
// the CTAs of one cluster.
NRG_DEV void fence_cluster() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }

// One cluster of kChaseCTAs CTAs per block; warp w of CTA r (global warp g = r*kChaseWarps + w)
// runs sweeps g, g + G, ... with G = kChaseCTAs * kChaseWarps. Step j of sweep i waits until
// sweep i-1 has finished step j+2: step j of sweep i touches rows i+1+(j-1)kBand ..
// i+1+(j+2)kBand-1 at most, and every step of sweep i-1 from step j+3 on touches only rows
// below them (the last row sweep i's step reaches is the column that sweep i-1's step j+3
// clears, whose entries that step stores in another column). Progress per warp, in its CTA's
// shared memory (read by the other CTAs through distributed shared memory): key(i, c) =
// i*(J+1) + c after c steps of sweep i (c = J when the sweep is done), monotone; the band
// stores are fenced at cluster scope before the key is published, and the reader fences
// after it sees the key. Waits are bounded: when one runs out, its CTA stops and marks the
// block.
__global__ void __launch_bounds__(32 * kChaseWarps) band_chase_kernel(const BandBlock* __restrict__ blocks) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const BandBlock B = blocks[blockIdx.x / kChaseCTAs];
  const int n = B.n, J = B.J, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = kChaseCTAs * kChaseWarps, gw = rank * kChaseWarps + warp;
  __shared__ volatile int prog[kChaseWarps];
  __shared__ volatile int abort_flag;
  __shared__ double vsh[kChaseWarps][kBand], wsh[kChaseWarps][kBand];
  extern __shared__ __align__(16) double ltsm[];  // kChaseWarps x 32 x 33
  double* lt = ltsm + (size_t)warp * kBand * (kBand + 1);
  // the final diagonal block [jfin, n) of S into the band (its distances <= kBand)
  const int nfin = (n - B.jfin) * (kBand + 1);
  for (int idx = rank * blockDim.x + tid; idx < nfin; idx += kChaseCTAs * blockDim.x) {
    const int c = B.jfin + idx / (kBand + 1), t = idx % (kBand + 1);
    if (c + t < n) B.BND[(size_t)c * kLDB + t] = B.S[(size_t)(c + t) * B.lds + c];
  }
  if (tid < kChaseWarps) prog[tid] = -1;
  if (tid == 0) abort_flag = 0;
  cl.sync();
  const int nsw = band_nsweeps(n);
  bool stop = false;  // warp-uniform
  for (int i = gw; i < nsw && !stop; i += G) {
    const int ns = band_nsteps(n, i);
    for (int j = 0; j < ns; j++) {
      if (i > 0) {
        const int gp = (i - 1) % G;
        volatile int* pp = cl.map_shared_rank(const_cast<int*>(prog), gp / kChaseWarps) + gp % kChaseWarps;
        const int need = (i - 1) * (J + 1) + min(j + 3, J);
        int ok = 1;
        if (lane == 0) {
          long long it = 0;
          while (*pp < need) {
            if (abort_flag) break;
            if (++it > (1LL << 24)) {
              abort_flag = 1;
              break;
            }
            __nanosleep(64);
          }
          ok = *pp >= need;
        }
        ok = __shfl_sync(kFull, ok, 0);
        if (!ok) {
          stop = true;
          break;
        }
        fence_cluster();
      }
      chase_step(B.BND, B.V2, B.tau2, n, J, i, j, lane, vsh[warp], wsh[warp], lt);
      __syncwarp();
      fence_cluster();
      if (lane == 0) prog[warp] = i * (J + 1) + (j + 1 == ns ? J : j + 1);
    }
  }
  cl.sync();  // every sweep is done (or stopped) and no CTA reads another's progress any more
  if (abort_flag && tid == 0) *B.info = 1;  // the chase did not finish: not converged, no result
  if (rank != 0) return;
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

// The window of group (g, j) covers rows rs .. rs+62 of the eigenvector components with
// rs = g*kGrp + 1 + j*kBand, so the windows of steps j and j+1 overlap in 31 columns: the
// window stays in shared memory along j (its first kBand columns are written back when it
// moves on), and the loads of the next group (its V, T and the kBand new window columns) are
// issued into registers before the current group's products, so that their latency overlaps
// the tensor-core work.
NRG_DEV double q2_v(const BandBlock& B, int g, int j, int q, int t, int nm) {
  return q < nm ? B.V2[((size_t)(g * kGrp + q) * B.J + j) * kBand + t] : 0.0;
}

__global__ void __launch_bounds__(256) band_q2_apply_kernel(const BandBlock* __restrict__ blocks) {
  const BandBlock B = blocks[blockIdx.y];
  const int n = B.n, J = B.J;
  const int e0 = blockIdx.x * kQ2Rows;
  if (e0 >= n || J == 0) return;
  const int ne = min(kQ2Rows, n - e0);
  extern __shared__ __align__(16) double q2sm[];
  double* W = q2sm;                  // 64 x kLW: the window Zt[e0 .., rs ..]
  double* V = W + 64 * kLW;          // 32 x kLW: row q = reflector q over the window's columns
  double* T = V + 32 * kLW;          // 32 x kLX
  double* X = T + 32 * kLX;          // 64 x kLX
  double* X2 = X + 64 * kLX;         // 64 x kLX
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int fr = lane >> 2, fc = lane & 3;
  const int rb = (warp >> 1) * 16;  // the warp's 16 rows of the window
  double* Z = B.evecs + (size_t)e0 * n;
  for (int idx = tid; idx < 32 * kLW; idx += 256) V[idx] = 0.0;  // off the parallelogram: zero for good
  // per-thread prefetch registers: 4 reflector entries, 4 T entries, 8 window entries
  double pv[4], pt[4], pw[8];
  auto prefetch = [&](int g, int j, int nm, int col0) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int idx = tid + 256 * k, q = idx >> 5, t = idx & 31;
      pv[k] = q2_v(B, g, j, q, t, nm);
      pt[k] = B.T2[((size_t)g * J + j) * kGrp * kGrp + idx];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int idx = tid + 256 * k, e = idx >> 5, c = idx & 31;
      const int gc = col0 + c;
      pw[k] = (e < ne && gc < n) ? Z[(size_t)e * n + gc] : 0.0;
    }
  };
  auto commit = [&](int wcol0) {  // prefetched V, T and window columns wcol0 .. wcol0+31 into place
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int idx = tid + 256 * k, q = idx >> 5, t = idx & 31;
      V[q * kLW + q + t] = pv[k];
      T[(idx >> 5) * kLX + (idx & 31)] = pt[k];
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int idx = tid + 256 * k, e = idx >> 5, c = idx & 31;
      if (wcol0 + c < 64) W[e * kLW + wcol0 + c] = pw[k];
    }
  };
  for (int g = band_ngroups(n) - 1; g >= 0; g--) {
    const int rs0 = g * kGrp + 1;
    int nm = group_members(n, g, 0);
    if (nm == 0) continue;
    // the first window: columns rs0 .. rs0+63 in two halves, V and T of step 0
    prefetch(g, 0, nm, rs0);
    __syncthreads();  // the previous pass's window is written back and free
    commit(0);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const int idx = tid + 256 * k, e = idx >> 5, c = idx & 31;
      const int gc = rs0 + 32 + c;
      W[e * kLW + 32 + c] = (e < ne && gc < n) ? Z[(size_t)e * n + gc] : 0.0;
    }
    for (int j = 0; j < J; j++) {
      const int rs = rs0 + j * kBand;
      const int nm_next = (j + 1 < J) ? group_members(n, g, j + 1) : 0;
      __syncthreads();  // window, V and T of (g, j) in place
      if (nm_next > 0) prefetch(g, j + 1, nm_next, rs + 64);
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
      // W -= X2 V (64 x 64, K = 32): warp tile 16 x 32, in place
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
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int jj = 0; jj < 4; jj++)
#pragma unroll
            for (int h = 0; h < 2; h++) W[(rb + 8 * i + fr) * kLW + cb + 8 * jj + 2 * fc + h] -= acc[i][jj][h];
      }
      __syncthreads();
      // the window's first kBand columns are final for this pass; the rest moves to the front
      const int ncols = nm_next > 0 ? 32 : 64;
      for (int idx = tid; idx < 64 * ncols; idx += 256) {
        const int e = idx / ncols, c = idx % ncols;
        if (e < ne && rs + c < n) Z[(size_t)e * n + rs + c] = W[e * kLW + c];
      }
      if (nm_next == 0) break;
      __syncthreads();
      for (int idx = tid; idx < 64 * 32; idx += 256) {
        const int e = idx >> 5, c = idx & 31;
        W[e * kLW + c] = W[e * kLW + 32 + c];
      }
      __syncthreads();  // the shift has read columns 32..63 before they are replaced
      commit(32);  // columns 32..63 of the next window, its V (zero rows for non-members) and T
      nm = nm_next;
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

cudaError_t band_panel_launch(const BandBlock* d_blocks, int nactive, int j0, int mmax, cudaStream_t s) {
  if (nactive <= 0) return cudaSuccess;
  // CTAs per block: enough that a share of the panel (kBand rows) fits 160 KB of shared memory
  int PC = 2;
  while (PC < 16 && (size_t)kBand * ((mmax + PC - 1) / PC + 1) * sizeof(double) > 160 * 1024) PC *= 2;
  const int chunk = (mmax + PC - 1) / PC;
  const size_t smem = sizeof(double) * ((size_t)kBand * (chunk + 1) + 2 + kBand + kPanelPairs + 64);
  cudaError_t err = cudaFuncSetAttribute(band_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err == cudaSuccess && PC > 8)
    err = cudaFuncSetAttribute(band_panel_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (err != cudaSuccess) return err;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nactive * PC));
  cfg.blockDim = dim3(kPanelThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)PC;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, band_panel_kernel, d_blocks, j0, chunk);
}

cudaError_t band_chase_launch(const BandBlock* d_blocks, int nblk, cudaStream_t s) {
  if (nblk <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * kChaseWarps * kBand * (kBand + 1);
  cudaError_t err = cudaFuncSetAttribute(band_chase_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return err;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(nblk * kChaseCTAs));
  cfg.blockDim = dim3(32 * kChaseWarps);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)kChaseCTAs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, band_chase_kernel, d_blocks);
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
