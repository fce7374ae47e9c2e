"""Host-side mirror of the reference interfaces of the NRG step core, over the C-ABI.

The names and argument meanings follow NRG Ljubljana's C++ host code:

* ``diagonalise(m, diag, diagratio)``          c++/diag.hpp:261-292 (real blocks)
* ``diagonalisations(blocks, ...)``             c++/core.hpp:90-120 (one batched call per step)
* ``product`` / ``transform`` / ``rotate``      c++/numerics_ublas.hpp:108-140
* ``gemm3_batch``                               all GEMM leaves of one recalculation in one call
* ``Bins.loggrid``                              c++/bins.hpp:61-100
* ``spec_accumulate``                           Algo_DMNRG / Algo_FDMgt / Algo_FDMls ::calc over all
                                                subspace pairs of a step (c++/algo.hpp:55-67)

Host (numpy) arguments go through the ``*_host`` entry points (copy in, compute on the
GPU, copy out); device arguments are torch CUDA tensors of dtype float64 whose
``data_ptr()`` is handed to the library. Nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import Bins as _BinsC, Gemm3, NRGError, SpecPair, SpecParams, check

_contexts = {}


class Context:
    """Per-device context: workspace arena and descriptor staging (nrg_create)."""

    def __init__(self, device: int = 0, workspace_limit: int = 0):
        self.lib = _lib.load()
        self.ptr = C.c_void_p()
        check(self.lib.nrg_create(C.byref(self.ptr), device, workspace_limit), "nrg_create")
        self.device = device

    def profile(self, enable: bool = True) -> None:
        """Start (reset) or stop per-phase CUDA-event timing (nrg_profile)."""
        check(self.lib.nrg_profile(self.ptr, int(enable)), "nrg_profile")

    def profile_read(self) -> dict:
        """{phase: (ms, launches)} since the last profile(True) (nrg_profile_read)."""
        arr = (_lib.PhaseStat * 32)()
        k = check(self.lib.nrg_profile_read(self.ptr, arr, 32), "nrg_profile_read")
        return {arr[i].name.decode(): (arr[i].ms, int(arr[i].launches)) for i in range(k)}

    @property
    def tuning(self) -> dict:
        """The eigensolver's launch parameters (nrg_get_tuning)."""
        t = _lib.Tuning()
        check(self.lib.nrg_get_tuning(self.ptr, C.byref(t)), "nrg_get_tuning")
        return {k: getattr(t, k) for k, _ in _lib.Tuning._fields_}

    def set_tuning(self, **kw) -> None:
        """Change some of the launch parameters (nrg_set_tuning; the library checks ranges)."""
        cur = self.tuning
        cur.update(kw)
        t = _lib.Tuning(**cur)
        check(self.lib.nrg_set_tuning(self.ptr, C.byref(t)), "nrg_set_tuning")

    def trim(self) -> None:
        """Give the context's device memory back (nrg_trim); later calls allocate again."""
        check(self.lib.nrg_trim(self.ptr), "nrg_trim")

    def close(self):
        if self.ptr:
            self.lib.nrg_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def context(device: int = 0) -> Context:
    """The process's context on `device`, created at first use with the autotuned launch
    parameters of that device model when a table for it is present (autotune.load_table)."""
    if device not in _contexts:
        ctx = Context(device)
        from .autotune import load_table
        table = load_table(device)
        if table:
            ctx.set_tuning(**table)
        _contexts[device] = ctx
    return _contexts[device]


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(None)
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


# ---------------------------------------------------------------- diagonalisation
@dataclass
class RawEigen:
    """Eigenvalues ascending and eigenvectors as rows (c++/eigen.hpp:180-199)."""
    val: np.ndarray
    vec: np.ndarray


def is_matrix_upper(m: np.ndarray) -> bool:
    """c++/numerics.hpp:140-146: square, lower triangle zero to 1e-12."""
    if m.ndim != 2 or m.shape[0] != m.shape[1]:
        return False
    low = np.tril(m, -1)
    return bool(np.all(np.abs(low) < 1e-12))


def diagonalisations(blocks: Sequence[np.ndarray], ctx: Optional[Context] = None, stream=None,
                     check_upper: bool = True) -> List[RawEigen]:
    """All blocks of one NRG step in one batched GPU call (host arrays in and out).

    Each block is n x n row-major with its upper triangle set, as built by hamiltonian()
    (c++/core.hpp:72-88); the lower triangle is ignored. Raises RuntimeError with the
    reference's message when a block fails (INFO != 0, c++/diag.hpp:80).
    """
    ctx = ctx or context()
    nb = len(blocks)
    if nb == 0:
        return []
    mats = []
    for b in blocks:
        m = np.ascontiguousarray(b, dtype=np.float64)
        if check_upper and not is_matrix_upper(m):
            raise AssertionError("is_matrix_upper(m) failed")  # my_assert, c++/diag.hpp:265
        mats.append(m)
    n = (C.c_int * nb)(*[m.shape[0] for m in mats])
    vals = [np.empty(m.shape[0]) for m in mats]
    vecs = [np.empty_like(m) for m in mats]
    H = (C.c_void_p * nb)(*[m.ctypes.data for m in mats])
    E = (C.c_void_p * nb)(*[v.ctypes.data for v in vals])
    V = (C.c_void_p * nb)(*[v.ctypes.data for v in vecs])
    info = (C.c_int * nb)()
    rc = ctx.lib.nrg_diag_batch_host(ctx.ptr, nb, n, H, E, V, info, _stream_ptr(stream))
    if rc < 0:
        raise NRGError(rc, "nrg_diag_batch_host")
    if rc > 0:
        bad = [i for i in range(nb) if info[i] != 0]
        raise RuntimeError(f"dsyev failed. INFO={info[bad[0]]} (block {bad[0]}, {len(bad)} blocks)")
    return [RawEigen(v, z) for v, z in zip(vals, vecs)]


def diagonalise(m: np.ndarray, diag: str = "dsyev", diagratio: float = 1.0, ctx: Optional[Context] = None) -> RawEigen:
    """diagonalise() of c++/diag.hpp:261-292 for one real block.

    diag in {"dsyev", "dsyevd", "default"} computes all pairs; "dsyevr" with
    diagratio < 1 returns the ceil(diagratio * dim) lowest pairs (c++/diag.hpp:118-130).
    """
    if diag not in ("dsyev", "dsyevd", "default", "dsyevr"):
        raise ValueError(f"unsupported diag={diag} for real matrices")
    r = diagonalisations([m], ctx)[0]
    if diag == "dsyevr" and diagratio != 1.0:
        M = min(max(int(math.ceil(diagratio * len(r.val))), 1), len(r.val))
        r = RawEigen(r.val[:M].copy(), r.vec[:M].copy())
    return r


def diag_batch_device(H, evals, evecs, ctx: Optional[Context] = None, stream=None) -> np.ndarray:
    """Batched eigensolve on device tensors (lists of torch CUDA float64 tensors).

    H[b] (n x n, upper triangle read) is overwritten; evals[b] (n) and evecs[b] (n x n)
    receive the result. Returns the per-block status words (0 = ok).
    """
    ctx = ctx or context()
    nb = len(H)
    n = (C.c_int * nb)(*[int(h.shape[0]) for h in H])
    Hp = (C.c_void_p * nb)(*[h.data_ptr() for h in H])
    Ep = (C.c_void_p * nb)(*[e.data_ptr() for e in evals])
    Vp = (C.c_void_p * nb)(*[v.data_ptr() for v in evecs])
    info = (C.c_int * nb)()
    rc = ctx.lib.nrg_diag_batch(ctx.ptr, nb, n, Hp, Ep, Vp, info, _stream_ptr(stream))
    if rc < 0:
        raise NRGError(rc, "nrg_diag_batch")
    return np.array(info[:], dtype=np.int32)


# ---------------------------------------------------------------- GEMM leaves
def _ptr_ld(x) -> Tuple[int, int]:
    """(address, leading dimension) of a 2-D row-major view (numpy or torch)."""
    if hasattr(x, "data_ptr"):
        if x.dim() != 2 or x.stride(1) != 1:
            raise ValueError("expected a 2-D view with unit column stride")
        return x.data_ptr(), x.stride(0)
    if x.ndim != 2 or x.strides[1] != 8 or x.dtype != np.float64:
        raise ValueError("expected a 2-D float64 view with unit column stride")
    return x.ctypes.data, x.strides[0] // 8


def gemm3(M, factor, A, O, B, transA=False, transB=True) -> Gemm3:
    """Descriptor of M += factor * op(A) * O * op(B) (O may be None for the identity)."""
    mp, ldm = _ptr_ld(M)
    ap, lda = _ptr_ld(A)
    bp, ldb = _ptr_ld(B)
    rows, cols = int(M.shape[0]), int(M.shape[1])
    ka = int(A.shape[0] if transA else A.shape[1])
    kb = int(B.shape[1] if transB else B.shape[0])
    op = ldo = 0
    if O is not None:
        op, ldo = _ptr_ld(O)
        if tuple(O.shape) != (ka, kb):
            raise ValueError(f"O shape {tuple(O.shape)} != ({ka}, {kb})")
    elif ka != kb:
        raise ValueError("identity O needs ka == kb")
    if (A.shape[1] if transA else A.shape[0]) != rows or (B.shape[0] if transB else B.shape[1]) != cols:
        raise ValueError("shape mismatch")
    return Gemm3(mp, ldm, ap, lda, op, ldo, bp, ldb, rows, cols, ka, kb, int(transA), int(transB), float(factor))


def gemm3_batch(terms: Sequence[Gemm3], host: bool, ctx: Optional[Context] = None, stream=None) -> None:
    ctx = ctx or context()
    arr = (Gemm3 * len(terms))(*terms)
    f = ctx.lib.nrg_gemm3_batch_host if host else ctx.lib.nrg_gemm3_batch
    check(f(ctx.ptr, len(terms), arr, _stream_ptr(stream)), "nrg_gemm3_batch")


def gemm3_batch_array(terms: np.ndarray, ctx: Optional[Context] = None, stream=None) -> None:
    """nrg_gemm3_batch on a numpy record array of GEMM3_DTYPE (device pointers)."""
    ctx = ctx or context()
    if terms.dtype != _lib.GEMM3_DTYPE or not terms.flags.c_contiguous:
        raise ValueError("terms must be a contiguous GEMM3_DTYPE array")
    if len(terms) == 0:
        return
    check(ctx.lib.nrg_gemm3_batch(ctx.ptr, len(terms), terms.ctypes.data_as(C.POINTER(Gemm3)), _stream_ptr(stream)),
          "nrg_gemm3_batch")


def hamiltonian_batch(n: Sequence[int], H: Sequence[int], pieces: np.ndarray, ctx: Optional[Context] = None,
                      stream=None) -> None:
    """nrg_hamiltonian_batch: blocks n[b] at device addresses H[b], pieces a HPIECE_DTYPE array."""
    ctx = ctx or context()
    if pieces.dtype != _lib.HPIECE_DTYPE or not pieces.flags.c_contiguous:
        raise ValueError("pieces must be a contiguous HPIECE_DTYPE array")
    nb = len(n)
    n_c = (C.c_int * nb)(*[int(x) for x in n])
    H_c = (C.c_void_p * nb)(*[int(x) for x in H])
    check(ctx.lib.nrg_hamiltonian_batch(ctx.ptr, nb, n_c, H_c, len(pieces),
                                        pieces.ctypes.data_as(C.POINTER(_lib.HPiece)), _stream_ptr(stream)),
          "nrg_hamiltonian_batch")


def diag_batch_ptrs(n: Sequence[int], H: Sequence[int], evals: Sequence[int], evecs: Sequence[int],
                    ctx: Optional[Context] = None, stream=None) -> np.ndarray:
    """nrg_diag_batch on raw device addresses; returns the per-block status words."""
    ctx = ctx or context()
    nb = len(n)
    n_c = (C.c_int * nb)(*[int(x) for x in n])
    Hp = (C.c_void_p * nb)(*[int(x) for x in H])
    Ep = (C.c_void_p * nb)(*[int(x) for x in evals])
    Vp = (C.c_void_p * nb)(*[int(x) for x in evecs])
    info = (C.c_int * nb)()
    rc = ctx.lib.nrg_diag_batch(ctx.ptr, nb, n_c, Hp, Ep, Vp, info, _stream_ptr(stream))
    if rc < 0:
        raise NRGError(rc, "nrg_diag_batch")
    return np.array(info[:], dtype=np.int32)


def _is_host(x) -> bool:
    return not hasattr(x, "data_ptr")


def product(M, factor, A, B, ctx=None, stream=None) -> None:
    """M += factor * A * B^T (c++/numerics_ublas.hpp:108-116)."""
    if A.shape[0] * A.shape[1] == 0 or B.shape[0] * B.shape[1] == 0:
        return
    gemm3_batch([gemm3(M, factor, A, None, B)], _is_host(M), ctx, stream)


def transform(M, factor, A, O, B, ctx=None, stream=None) -> None:
    """M += factor * A * O * B^T (c++/numerics_ublas.hpp:119-128)."""
    if A.shape[0] * A.shape[1] == 0 or B.shape[0] * B.shape[1] == 0:
        return
    gemm3_batch([gemm3(M, factor, A, O, B)], _is_host(M), ctx, stream)


def rotate(M, factor, U, O, ctx=None, stream=None) -> None:
    """M += factor * U^T * O * U (c++/numerics_ublas.hpp:130-140)."""
    if U.shape[0] * U.shape[1] == 0:
        return
    gemm3_batch([gemm3(M, factor, U, O, U, transA=True, transB=False)], _is_host(M), ctx, stream)


# ---------------------------------------------------------------- spectral accumulation
@dataclass
class BinGrid:
    """Standard log grid of c++/bins.hpp:61-100 for one sign half."""
    log10emin: float
    log10emax: float
    bins: int
    discard_immediately: float = 0.0

    @classmethod
    def from_limits(cls, emin: float, emax: float, bins: int, discard_immediately: float = 0.0) -> "BinGrid":
        return cls(math.floor(math.log10(emin)), math.ceil(math.log10(emax)), bins, discard_immediately)

    @property
    def nbins(self) -> int:
        return int((self.log10emax - self.log10emin) * self.bins + 1.0)

    def c(self) -> _BinsC:
        return _BinsC(self.log10emin, self.log10emax, self.bins, self.nbins, self.discard_immediately)

    def energies(self) -> np.ndarray:
        out = np.zeros(self.nbins)
        b = self.c()
        _lib.load().nrg_bins_grid(C.byref(b), out.ctypes.data_as(C.POINTER(C.c_double)))
        return out


def spec_pair(Ei, Ej, op1, op2, ki, kj, factor, rho_i=None, rho_j=None) -> SpecPair:
    """Descriptor of one subspace pair (Ii, Ij) on device tensors; see include/nrg_b200.h."""
    p1, ld1 = _ptr_ld(op1)
    p2, ld2 = _ptr_ld(op2)
    ri = rj = 0
    ldri = ldrj = 0
    rdi = rdj = 0
    if rho_i is not None:
        ri, ldri = _ptr_ld(rho_i)
        rdi = int(rho_i.shape[0])
    if rho_j is not None:
        rj, ldrj = _ptr_ld(rho_j)
        rdj = int(rho_j.shape[0])
    return SpecPair(Ei.data_ptr(), Ej.data_ptr(), p1, ld1, p2, ld2, ri, ldri, rj, ldrj, int(Ei.shape[0]), int(ki),
                    int(Ej.shape[0]), int(kj), rdi, rdj, float(factor))


def spec_accumulate(algo: int, pairs: Sequence[SpecPair], grid: BinGrid, pos, neg, sign: int = -1, T: float = 0.0,
                    wnf: float = 0.0, Emin: float = 0.0, Emax: float = 0.0, ctx=None, stream=None) -> None:
    """Accumulate the spectral weights of all pairs into pos/neg (device tensors, +=)."""
    ctx = ctx or context()
    arr = (SpecPair * len(pairs))(*pairs)
    prm = SpecParams(algo, sign, T, wnf, Emin, Emax)
    b = grid.c()
    check(ctx.lib.nrg_spec_accumulate(ctx.ptr, len(pairs), arr, C.byref(prm), C.byref(b), C.c_void_p(pos.data_ptr()),
                                      C.c_void_p(neg.data_ptr()), _stream_ptr(stream)), "nrg_spec_accumulate")


def spec_accumulate_array(algo: int, pairs: np.ndarray, grid: BinGrid, pos, neg, sign: int = -1, T: float = 0.0,
                          wnf: float = 0.0, Emin: float = 0.0, Emax: float = 0.0, ctx=None, stream=None) -> None:
    """nrg_spec_accumulate on a numpy record array of SPECPAIR_DTYPE (device pointers)."""
    ctx = ctx or context()
    if pairs.dtype != _lib.SPECPAIR_DTYPE or not pairs.flags.c_contiguous:
        raise ValueError("pairs must be a contiguous SPECPAIR_DTYPE array")
    prm = SpecParams(algo, sign, T, wnf, Emin, Emax)
    b = grid.c()
    check(ctx.lib.nrg_spec_accumulate(ctx.ptr, len(pairs), pairs.ctypes.data_as(C.POINTER(SpecPair)), C.byref(prm),
                                      C.byref(b), C.c_void_p(pos.data_ptr()), C.c_void_p(neg.data_ptr()),
                                      _stream_ptr(stream)), "nrg_spec_accumulate")


def spec_accumulate_mats_array(algo: int, pairs: np.ndarray, mats: int, re, im, sign: int, T: float, wnf: float,
                               ctx=None, stream=None) -> None:
    """nrg_spec_accumulate_mats (NRG_SPEC_FDMMATS, NRG_SPEC_FTMATS or NRG_SPEC_DMNRG on the
    Matsubara axis) on a numpy record array of SPECPAIR_DTYPE (device pointers); re, im: device
    tensors of mats doubles, accumulated."""
    ctx = ctx or context()
    if pairs.dtype != _lib.SPECPAIR_DTYPE or not pairs.flags.c_contiguous:
        raise ValueError("pairs must be a contiguous SPECPAIR_DTYPE array")
    prm = SpecParams(algo, sign, T, wnf, 0.0, 0.0)
    check(ctx.lib.nrg_spec_accumulate_mats(ctx.ptr, len(pairs), pairs.ctypes.data_as(C.POINTER(SpecPair)),
                                           C.byref(prm), int(mats), C.c_void_p(re.data_ptr()),
                                           C.c_void_p(im.data_ptr()), _stream_ptr(stream)), "nrg_spec_accumulate_mats")


def broaden(e: np.ndarray, w: np.ndarray, mesh: np.ndarray, alpha: float, omega0: float, ctx=None,
            stream=None) -> np.ndarray:
    """Log-Gaussian broadening (nrg_broaden) of peaks (e, w) onto the mesh; host arrays in
    and out, computed on the device."""
    import torch
    ctx = ctx or context()
    dev = torch.device("cuda", ctx.device)
    te = torch.from_numpy(np.ascontiguousarray(e, dtype=np.float64)).to(dev)
    tw = torch.from_numpy(np.ascontiguousarray(w, dtype=np.float64)).to(dev)
    tm = torch.from_numpy(np.ascontiguousarray(mesh, dtype=np.float64)).to(dev)
    out = torch.empty(len(mesh), dtype=torch.float64, device=dev)
    check(ctx.lib.nrg_broaden(ctx.ptr, len(e), C.c_void_p(te.data_ptr()), C.c_void_p(tw.data_ptr()), len(mesh),
                              C.c_void_p(tm.data_ptr()), float(alpha), float(omega0), C.c_void_p(out.data_ptr()),
                              _stream_ptr(stream)), "nrg_broaden")
    return out.cpu().numpy()
