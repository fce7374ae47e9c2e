/* nrg_b200.h -- C-ABI of the B200 (sm_100a) NRG step core.
 *
 * Drop-in boundary for the data-parallel hot path of one NRG iteration of NRG Ljubljana:
 * the diagonalisation of every symmetry-subspace block, the recalculation of irreducible
 * matrix elements (U^T O U contractions), the density-matrix rotations and the DM-NRG /
 * FDM spectral-weight accumulation into log-spaced bins. All arithmetic is FP64.
 *
 * Conventions (those of the reference):
 *   - matrices are dense ROW-major with an explicit leading dimension (elements between
 *     rows); strided views such as the ancestor blocks U(i) of recalc.hpp are expressed
 *     by a pointer to their first element plus the leading dimension of the parent;
 *   - a diagonalised block returns its eigenvalues ascending and its eigenvectors as ROWS
 *     (vec(r, j) = component j of eigenvector r), c++/diag.hpp:41-48;
 *   - entry points without the _host suffix take DEVICE pointers and are asynchronous on
 *     `stream` (a cudaStream_t, NULL = legacy default stream); the _host variants take
 *     HOST pointers, copy in, compute and copy out, and return when the results are in
 *     host memory.
 * Return codes: NRG_OK, a negative NRG_ERR_* code, or (diagonalisation) the number of
 * blocks whose per-block status word is non-zero. nrg_last_error() gives the message of
 * the last failure on the calling thread. No entry point falls back to the CPU.
 */
#ifndef NRG_B200_H
#define NRG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NRG_B200_VERSION 2

#define NRG_OK 0
#define NRG_ERR_ARG (-1)    /* invalid argument (sizes, null pointers, shapes) */
#define NRG_ERR_CUDA (-2)   /* a CUDA runtime call or a kernel launch failed */
#define NRG_ERR_OOM (-3)    /* device workspace could not be allocated within the budget */
#define NRG_ERR_NODEV (-4)  /* no usable sm_100 device */

#if defined(__GNUC__)
#define NRG_API __attribute__((visibility("default")))
#else
#define NRG_API
#endif

typedef struct nrg_ctx nrg_ctx;

NRG_API int nrg_version(void);
NRG_API const char* nrg_last_error(void);

/* Per-run context: device, device workspace (grown on demand up to workspace_limit bytes,
 * 0 = 90% of the free device memory at creation, and never past the memory free at the
 * time less a reserve of 2 GiB or 2% of the device: larger batches are solved in chunks),
 * descriptor staging. One context may
 * be used from one host thread at a time. Calls on one context may name different
 * streams: each call's work is ordered after the previous call's (an event recorded on
 * the previous call's stream), because all calls share the context's descriptor staging
 * and workspace. Independent work on several streams at once needs one context each. */
NRG_API int nrg_create(nrg_ctx** ctx, int device, size_t workspace_limit);
NRG_API int nrg_destroy(nrg_ctx* ctx);
/* Gives the context's device memory back (workspace arena, host-block ring, descriptor
 * staging) after synchronising the device; later calls allocate again as needed. */
NRG_API int nrg_trim(nrg_ctx* ctx);

/* Launch parameters of the batched eigensolver, chosen per device by the autotuner
 * (nrgljubljana_b200/autotune.py) from timed sweeps; the defaults are its result on B200.
 *   small_max_n    blocks up to this order are solved whole in the shared memory of one
 *                  CTA (32..96)
 *   mid_max_n      larger blocks up to this order are reduced to tridiagonal form in the
 *                  shared memory of one CTA (small_max_n..236)
 *   cluster_max_n  larger blocks up to this order are reduced in the distributed shared
 *                  memory of a thread-block cluster when the clusters fit the SMs at once
 *                  (mid_max_n..640); larger blocks stream their trailing matrix from HBM
 *   reduction_ctas_per_sm  most CTAs of the streaming reduction kernel per SM (1, 2 or 3;
 *                  default 3), used when the batch's streamed blocks fill three waves of them
 *                  (fewer otherwise: a batch of few large blocks is bound by its largest)
 *   band_min_n     blocks of at least this order, when at most band_max_blocks of them are
 *                  in a batch, take the two-stage reduction (dense -> band on the FP64
 *                  tensor cores, band -> tridiagonal by bulge chasing); 0 = never; default 3072
 *   band_max_blocks  see band_min_n (few large blocks: the regime where the one-stage
 *                  reduction's per-column chain bounds the step); default 64 */
typedef struct nrg_tuning {
  int small_max_n;
  int mid_max_n;
  int cluster_max_n;
  int reduction_ctas_per_sm;
  int band_min_n;
  int band_max_blocks;
} nrg_tuning;
NRG_API int nrg_get_tuning(nrg_ctx* ctx, nrg_tuning* out);
NRG_API int nrg_set_tuning(nrg_ctx* ctx, const nrg_tuning* in);

/* ------------------------------------------------------------------ diagonalisation
 * Replaces diagonalise() (c++/diag.hpp:261-292) with diag=dsyev|dsyevd|default for real
 * matrices, and the per-step batch loop diagonalisations() / diagonalisations_OpenMP()
 * (c++/core.hpp:90-120): all nblk blocks of a step in one call.
 *   n[b]       order of block b (host array), 1 <= n[b] <= NRG_DIAG_MAX_N
 *   H[b]       n x n row-major, upper triangle read (lower ignored); CONSUMED (overwritten),
 *              as the reference consumes its argument (c++/diag.hpp:259-260)
 *   evals[b]   n doubles, ascending
 *   evecs[b]   n x n row-major, row r = eigenvector of evals[b][r]
 *   info       host array of nblk status words: 0 ok; -2 non-finite input; > 0 the
 *              tridiagonal iteration did not converge (the reference's INFO != 0)
 * H, evals, evecs are host arrays of device pointers; evecs[b] must not alias H[b]. */
#define NRG_DIAG_MAX_N 10240
NRG_API int nrg_diag_batch(nrg_ctx* ctx, int nblk, const int* n, double* const* H, double* const* evals,
                   double* const* evecs, int* info, void* stream);

/* Same with host pointers for H[b], evals[b], evecs[b] (the call the reference's
 * diagonalise() makes with its ublas matrix); H[b] is left unchanged. The blocks stream
 * through a ring of at most three device slots in chunks of consecutive blocks (a chunk
 * holds about half of the batch, at most 32 GiB): the copy of chunk k+1 to the device
 * and of chunk k-1 back to the host overlap the solve of chunk k, on two copy streams of
 * the context. Page-locked host memory lets the copies run asynchronously; pageable
 * memory works too, with copies that do not overlap. Returns when every result is in host
 * memory. */
NRG_API int nrg_diag_batch_host(nrg_ctx* ctx, int nblk, const int* n, const double* const* H, double* const* evals,
                        double* const* evecs, int* info, void* stream);

/* ------------------------------------------------------------------ Hamiltonian assembly
 * Replaces hamiltonian() (c++/core.hpp:72-88) for all blocks of one step: the per-block
 * matrix initialisation of make_matrix() (c++/symmetry/sym-QS-impl.hpp:111-155) is given
 * as a list of pieces instead of being run per block on the host. Each H[b] (n[b] x n[b],
 * row-major, device) is cleared and the pieces with blk == b are added in the order given:
 *   NRG_HP_DIAG   H[r0+k][c0+k] += factor * src[k] + shift  for k < rows (src NULL: 0)
 *                 -- the ancestor energies scaled by sqrt(Lambda) (c++/core.hpp:79-82),
 *                 diag_function_impl (c++/matrix.hpp:67-78) and diag_offdiag_function
 *                 (c++/matrix.hpp:97-111)
 *   NRG_HP_BLOCK  H[r0+i][c0+j] += factor * src[i*ld + j]   (trans = 0)
 *                 H[r0+i][c0+j] += factor * src[j*ld + i]   (trans = 1, the conjugate
 *                 transpose of c++/matrix.hpp:48-52 for real matrices), i < rows, j < cols
 *                 -- offdiag_function_impl (c++/matrix.hpp:32-58)
 * Products and sums are rounded one by one (no fused multiply-add), so the result is
 * bit-identical to the reference's. The caller keeps every piece inside the upper
 * triangle, as the reference does; the strictly lower triangle is then zero, as
 * diagonalise() asserts (c++/diag.hpp:265). A non-finite factor is rejected as
 * offdiag_function() rejects it (c++/matrix.hpp:40-41). src pointers are device pointers;
 * n, H and pieces are host arrays. */
#define NRG_HP_DIAG 0
#define NRG_HP_BLOCK 1
typedef struct nrg_hpiece {
  int blk, kind;
  int r0, c0, rows, cols;
  int trans, pad_;
  int64_t ld;
  const double* src;
  double factor, shift;
} nrg_hpiece;
NRG_API int nrg_hamiltonian_batch(nrg_ctx* ctx, int nblk, const int* n, double* const* H, int npiece,
                                  const nrg_hpiece* pieces, void* stream);

/* ------------------------------------------------------------------ GEMM leaves
 * One term M += factor * op(A) * O * op(B), grouped by M. Expresses
 *   product   (c++/numerics_ublas.hpp:108-116): M += f A B^T         O = NULL, transB = 1
 *   transform (c++/numerics_ublas.hpp:119-128): M += f A O B^T       transB = 1
 *   rotate    (c++/numerics_ublas.hpp:130-140): M += f U^T O U       A = U, transA = 1, B = U
 * as used by recalc_general / recalc_f / recalc1_global (c++/recalc.hpp:52-122) and
 * cdmI (c++/dmnrg.hpp:55-80). op(A) is rows x ka, O is ka x kb (NULL means the identity,
 * ka == kb; ldo == 0 means a diagonal O given as its ka diagonal entries, ka == kb, as
 * the discarded-state sector of the FDM density matrix of init_rho_FDM,
 * c++/dmnrg.hpp:146-162, enters calc_fulldensitymatrix_iterN), op(B) is kb x cols. The
 * product O op(B) is formed first, as in the reference (for a diagonal O by scaling the
 * rows of op(B)). Terms with the same M are summed in the order given; distinct M regions must
 * not overlap. A term with rows, cols, ka or kb zero is skipped (finite_size checks of the
 * reference). Pointers are device pointers. The intermediates O op(B) (ka x cols each) live
 * in the context's workspace; when all of them do not fit in what it may hold, the call runs
 * in passes on the stream (whole groups of one M, or the terms of one group), and fails with
 * NRG_ERR_OOM only for a single term whose intermediate does not fit. */
typedef struct nrg_gemm3 {
  double* M;
  int64_t ldm;
  const double* A;
  int64_t lda;
  const double* O;
  int64_t ldo;
  const double* B;
  int64_t ldb;
  int rows, cols, ka, kb;
  int transA, transB;
  double factor;
} nrg_gemm3;

NRG_API int nrg_gemm3_batch(nrg_ctx* ctx, int nterm, const nrg_gemm3* terms, void* stream);
NRG_API int nrg_gemm3_batch_host(nrg_ctx* ctx, int nterm, const nrg_gemm3* terms, void* stream);

/* One transform term, M (rows x cols) += factor * A (rows x ka) * O (ka x kb) * B^T
 * (B is cols x kb; O = NULL means the identity, ka == kb), that allocates nothing.
 * Leading dimensions: ldm >= cols, lda >= ka, ldb >= kb and, with O, ldo >= kb (O is
 * always dense here: the diagonal O of nrg_gemm3 (ldo == 0) is rejected, as are A
 * transposed and B stored kb x cols; those terms need nrg_gemm3_batch).
 * This entry point has no counterpart in the reference. It is for callers that cannot call
 * cudaMalloc: a host thread that must not stall the device (cudaMalloc/cudaFree may
 * synchronise it), a plugin in a process whose device memory is already reserved by
 * another allocator, or code that may not own device memory. It needs no context: the
 * intermediate O * B^T is kept in a fixed device array of NRG_NOALLOC_SCRATCH_DOUBLES
 * doubles (8 MiB) that every GPU loading this library holds until the process exits, and
 * ka * cols beyond that limit is rejected with NRG_ERR_ARG. Pointers are device pointers on
 * the current device. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture. All calls share
 * the array: calls that overlap on the GPU (other streams, other host threads) race. */
#define NRG_NOALLOC_SCRATCH_DOUBLES (1 << 20)
NRG_API int nrg_transform_noalloc(double* M, int64_t ldm, const double* A, int64_t lda, const double* O,
                                  int64_t ldo, const double* B, int64_t ldb, int rows, int cols, int ka, int kb,
                                  double factor, void* stream);

/* ------------------------------------------------------------------ spectral accumulation
 * Replaces the per-pair calc() of Algo_DMNRG (c++/algo_DMNRG.hpp:29-52), Algo_FDMgt
 * (c++/algo_FDM.hpp:84-114) and Algo_FDMls (c++/algo_FDM.hpp:30-60), driven over all
 * subspace pairs of one step as BaseSpectrum::calc does (c++/algo.hpp:55-67), binned by
 * ChainBinning/Bins (c++/spectrum.hpp:19-28, c++/bins.hpp:95-132) on the standard log
 * grid. Weights are real (S = double). One pair (Ii, Ij) has
 *   op1, op2   dim_j x dim_i, row-major (rows: states of Ij, columns: states of Ii)
 *   Ei, Ej     energies (abs_zero for DMNRG, abs_G for FDM), ni and nj entries
 *   ki, kj     kept states (DMNRG: the loop ranges; FDM: K ranges, the rest is D)
 *   rho_i      DMNRG: rho(Ii) (ki x ki); FDM-gt: rhoFDM(Ii) (rdi x rdi); else unused
 *   rho_j      DMNRG: rho(Ij) (kj x kj); FDM-ls: rhoFDM(Ij) (rdj x rdj); else unused
 *   factor     ff(Ii, Ij)
 * algo: NRG_SPEC_DMNRG, NRG_SPEC_FDMGT, NRG_SPEC_FDMLS. pos/neg: device arrays of
 * bins.nbins doubles per sign half, ACCUMULATED (+=). */
#define NRG_SPEC_DMNRG 0
#define NRG_SPEC_FDMGT 1
#define NRG_SPEC_FDMLS 2

typedef struct nrg_spec_pair {
  const double* Ei;
  const double* Ej;
  const double* op1;
  int64_t ld1;
  const double* op2;
  int64_t ld2;
  const double* rho_i;
  int64_t ldri;
  const double* rho_j;
  int64_t ldrj;
  int ni, ki, nj, kj;
  int rdi, rdj;
  double factor;
} nrg_spec_pair;

typedef struct nrg_spec_params {
  int algo;
  int sign;      /* 1 bosonic, -1 fermionic (gf_sign) */
  double T;      /* temperature (FDM) */
  double wnf;    /* stats.wnfactor[step.ndx()] (FDM) */
  double Emin;   /* DMNRG window: step.scale() * P.getEmin() */
  double Emax;   /* DMNRG window: step.scale() * P.getEmax() */
} nrg_spec_params;

typedef struct nrg_bins {
  double log10emin;            /* floor(log10(emin)), c++/bins.hpp:67 */
  double log10emax;            /* ceil(log10(emax)),  c++/bins.hpp:68 */
  int bins;                    /* bins per decade (P.bins) */
  int nbins;                   /* (int)((log10emax - log10emin) * bins + 1), c++/bins.hpp:97 */
  double discard_immediately;  /* P.discard_immediately, c++/bins.hpp:105 */
} nrg_bins;

NRG_API int nrg_spec_accumulate(nrg_ctx* ctx, int npair, const nrg_spec_pair* pairs, const nrg_spec_params* params,
                        const nrg_bins* bins, double* pos, double* neg, void* stream);

/* Replaces the per-pair calc() of the Matsubara algorithms with their ChainMatsubara
 * accumulation (c++/spectrum.hpp:34-42, c++/matsubara.hpp:31-49): every term, weight w at
 * energy E = Ej - Ei, adds factor * w / (i w_n - E) to re[n] + i im[n] for n < mats
 * (ACCUMULATED), w_n = (2n+1) pi T for sign = -1 (fermionic) and 2n pi T for sign = +1
 * (bosonic). params->algo selects the terms:
 *   NRG_SPEC_FDMMATS  Algo_FDMmats (c++/algo_FDM.hpp:153-217): the terms of NRG_SPEC_FDMGT and
 *                     NRG_SPEC_FDMLS together (rho_i = rhoFDM(Ii) with rdi, rho_j = rhoFDM(Ij)
 *                     with rdj; abs_G energies; params->wnf)
 *   NRG_SPEC_FTMATS   Algo_FTmats (c++/algo_FT.hpp:50-91): over the pair's states (give the
 *                     kept x kept blocks, abs_zero energies), op1 op2 (e^{-Ei/T} - sign
 *                     e^{-Ej/T}) * params->wnf, wnf = 1 / Z_ft of the step
 *   NRG_SPEC_DMNRG    Algo_DMNRGmats (c++/algo_DMNRG.hpp:61-106): the DM-NRG weights of
 *                     nrg_spec_accumulate over kept x kept, without its energy window
 * For a bosonic operator the reference replaces the n = 0 term with |E| <= 1e-8 (WEIGHT_TOL)
 * by its limit, and so does this call: -w_gt / T for the FDM D x D term (w_gt its exp(-Ei/T)
 * part, c++/algo_FDM.hpp:178-188), -op1 op2 e^{-Ej/T} wnf / T for FT (c++/algo_FT.hpp:66-71),
 * -X op1 / T for DM-NRG (c++/algo_DMNRG.hpp:88-93). 1 <= mats <= 6144. */
#define NRG_SPEC_FDMMATS 3
#define NRG_SPEC_FTMATS 4
NRG_API int nrg_spec_accumulate_mats(nrg_ctx* ctx, int npair, const nrg_spec_pair* pairs,
                                     const nrg_spec_params* params, int mats, double* re, double* im, void* stream);

/* ------------------------------------------------------------------ timing
 * Per-phase device timing in the spirit of the reference's MemTime::time_it sections
 * (c++/time_mem.hpp:97-115): nrg_profile(ctx, 1) resets the counters and brackets every
 * later launch group with CUDA events on its stream; nrg_profile_read synchronises on
 * those events and returns one entry per phase that launched (name, total ms, number of
 * kernel launches). Launch counts are kept even when timing is off. */
/* Log-Gaussian broadening of a spectrum of delta peaks onto an energy mesh: replaces
 * SpectrumRealFreq::continuous() (c++/spectrum.hpp:168-196) with the kernel BR_NEW
 * (c++/spectral.hpp:42-70),
 *   out[k] = sum_s w[s] * BR_NEW(E[k], e[s], alpha, omega0),   k < nmesh, s < nspike.
 * Peaks of both signs and mesh points of both signs are given in one list each (the
 * reference's positive and negative halves). e, w, E, out are device arrays; out is
 * overwritten. The sum over peaks is taken in a fixed order. */
NRG_API int nrg_broaden(nrg_ctx* ctx, int nspike, const double* e, const double* w, int nmesh, const double* E,
                        double alpha, double omega0, double* out, void* stream);

typedef struct nrg_phase_stat {
  char name[24];
  double ms;
  long long launches;
} nrg_phase_stat;

NRG_API int nrg_profile(nrg_ctx* ctx, int enable);
NRG_API int nrg_profile_read(nrg_ctx* ctx, nrg_phase_stat* out, int max);

/* Energies of the log grid (c++/bins.hpp:95-100) for one sign half; returns nbins. */
NRG_API int nrg_bins_grid(const nrg_bins* bins, double* energies_host);

#ifdef __cplusplus
}
#endif

#endif /* NRG_B200_H */
