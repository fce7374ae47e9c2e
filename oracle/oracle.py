"""CPU oracle for the NRG step core -- TEST INFRASTRUCTURE ONLY.

Python face of ``oracle/nrg_oracle.cpp``, the plain-C++ restatement (over the host
OpenBLAS LAPACK) of NRG Ljubljana's hot path: ``diagonalise`` (c++/diag.hpp:62-172,
261-292), the GEMM leaves ``product``/``transform``/``rotate``
(c++/numerics_ublas.hpp:108-140), ``prod_fit`` (c++/numerics.hpp:283-306), ``Bins``
(c++/bins.hpp:61-132), ``ChainBinning`` (c++/spectrum.hpp:19-28), ``mergeNN2half``
(c++/spectrum.hpp:91-128), ``Algo_DMNRG::calc`` (c++/algo_DMNRG.hpp:29-52) and
``Algo_FDMgt/ls::calc`` (c++/algo_FDM.hpp:30-114).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this module, and only as the checker or the timed CPU reference.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++ + host OpenBLAS)."""
    src = os.path.join(_HERE, "nrg_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.oracle_blas_threads.argtypes = [C.c_int]
        L.oracle_blas_threads.restype = C.c_int
        L.oracle_diagonalise.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.oracle_diagonalise.restype = C.c_int
        L.oracle_diag_batch.argtypes = [C.c_int, _ip, _lp, _lp, _dp, _dp, _dp, C.c_int, C.c_int, _ip]
        L.oracle_diag_batch.restype = C.c_int
        L.oracle_is_unitary.argtypes = [C.c_int, C.c_int, _dp, C.c_double, C.c_double]
        L.oracle_is_unitary.restype = C.c_int
        L.oracle_product.argtypes = [C.c_int] * 3 + [C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.oracle_transform.argtypes = [C.c_int] * 4 + [C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                                        C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.oracle_rotate.argtypes = [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                    C.c_void_p, C.c_int]
        L.oracle_matmul.argtypes = [C.c_int] * 3 + [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.oracle_chit_weight.argtypes = [C.c_double] * 3
        L.oracle_chit_weight.restype = C.c_double
        L.oracle_loggrid.argtypes = [C.c_double, C.c_double, C.c_int, C.c_void_p]
        L.oracle_loggrid.restype = C.c_int
        L.oracle_chain_add.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_double, C.c_int, C.c_double, C.c_int,
                                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.oracle_windowfunction.argtypes = [C.c_double] * 4 + [C.c_int, C.c_double]
        L.oracle_windowfunction.restype = C.c_double
        L.oracle_merge_nn2half.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_double, C.c_double, C.c_double,
                                                              C.c_int, C.c_double, C.c_int]
        L.oracle_dmnrg_pair.argtypes = ([C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                         C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                         C.c_double, C.c_int, C.c_double, C.c_double]
                                        + [C.c_void_p] * 4 + [C.c_int, C.c_double, C.c_int, C.c_double])
        L.oracle_fdm_pair.argtypes = ([C.c_int] * 5 + [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                                       C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                                       C.c_double, C.c_double]
                                      + [C.c_void_p] * 4 + [C.c_int, C.c_double, C.c_int, C.c_double])
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def blas_threads(n: int = 0) -> int:
    return lib().oracle_blas_threads(n)


def diagonalise(h: np.ndarray, solver: str = "dsyev", ratio: float = 1.0):
    """diagonalise() of c++/diag.hpp:261-292 for one real block.

    ``h`` is n x n row-major with the upper triangle set (lower part ignored). Returns
    (eigenvalues ascending, eigenvectors as rows); raises RuntimeError on INFO != 0.
    """
    n = h.shape[0]
    H = np.ascontiguousarray(h, dtype=np.float64).copy()
    w = np.zeros(n)
    z = np.zeros((n, n))
    m = C.c_int(0)
    code = {"dsyev": 0, "default": 0, "dsyevd": 1, "dsyevr": 2}[solver]
    info = lib().oracle_diagonalise(n, H, w, z, code, ratio, C.byref(m))
    if info != 0:
        raise RuntimeError(f"{solver} failed. INFO={info}")
    M = m.value
    return w[:M].copy(), z[:M].copy()


def diag_batch(blocks, nthreads: int = 1, solver: str = "dsyev"):
    """OpenMP-over-blocks batch (c++/core.hpp:90-110); returns lists (evals, evecs)."""
    n = np.array([b.shape[0] for b in blocks], dtype=np.int32)
    moff = np.zeros(len(blocks), dtype=np.int64)
    voff = np.zeros(len(blocks), dtype=np.int64)
    if len(blocks) > 1:
        moff[1:] = np.cumsum(n.astype(np.int64) ** 2)[:-1]
        voff[1:] = np.cumsum(n.astype(np.int64))[:-1]
    H = np.concatenate([np.ascontiguousarray(b, dtype=np.float64).ravel() for b in blocks]) if blocks else np.zeros(1)
    V = np.zeros(max(1, int(n.astype(np.int64).sum())))
    Z = np.zeros_like(H)
    info = np.zeros(len(blocks), dtype=np.int32)
    code = {"dsyev": 0, "default": 0, "dsyevd": 1}[solver]
    bad = lib().oracle_diag_batch(len(blocks), n, moff, voff, H, V, Z, code, nthreads, info)
    if bad:
        raise RuntimeError(f"{bad} blocks failed: INFO={info[info != 0][:4]}")
    ev = [V[voff[b]:voff[b] + n[b]].copy() for b in range(len(blocks))]
    vec = [Z[moff[b]:moff[b] + n[b] * n[b]].reshape(n[b], n[b]).copy() for b in range(len(blocks))]
    return ev, vec


def diag_batch_packed(n: np.ndarray, moff: np.ndarray, voff: np.ndarray, H: np.ndarray, V: np.ndarray, Z: np.ndarray,
                      nthreads: int) -> int:
    """Packed-buffer batch used for timing (no per-block Python objects)."""
    info = np.zeros(len(n), dtype=np.int32)
    return lib().oracle_diag_batch(len(n), n, moff, voff, H, V, Z, 0, nthreads, info)


def is_unitary(vec: np.ndarray, norm_eps: float = 1e-12, ortho_eps: float = 1e-10) -> bool:
    v = np.ascontiguousarray(vec, dtype=np.float64)
    return bool(lib().oracle_is_unitary(v.shape[0], v.shape[1], v, norm_eps, ortho_eps))


def product(M: np.ndarray, factor: float, A: np.ndarray, B: np.ndarray) -> None:
    """M += factor * A * B^T (c++/numerics_ublas.hpp:108-116), in place."""
    if A.size == 0 or B.size == 0:
        return
    assert M.shape == (A.shape[0], B.shape[0]) and A.shape[1] == B.shape[1]
    lib().oracle_product(M.shape[0], M.shape[1], A.shape[1], factor, _ptr(A), A.shape[1], _ptr(B), B.shape[1],
                         _ptr(M), M.shape[1])


def transform(M: np.ndarray, factor: float, A: np.ndarray, O: np.ndarray, B: np.ndarray) -> None:
    """M += factor * A * O * B^T (c++/numerics_ublas.hpp:119-128), in place."""
    if A.size == 0 or B.size == 0:
        return
    assert M.shape == (A.shape[0], B.shape[0]) and A.shape[1] == O.shape[0] and O.shape[1] == B.shape[1]
    lib().oracle_transform(M.shape[0], M.shape[1], O.shape[0], O.shape[1], factor, _ptr(A), A.shape[1], _ptr(O),
                           O.shape[1], _ptr(B), B.shape[1], _ptr(M), M.shape[1])


def rotate(M: np.ndarray, factor: float, U: np.ndarray, O: np.ndarray) -> None:
    """M += factor * U^T * O * U (c++/numerics_ublas.hpp:130-140), in place."""
    if U.size == 0:
        return
    assert M.shape == (U.shape[1], U.shape[1]) and O.shape == (U.shape[0], U.shape[0])
    lib().oracle_rotate(U.shape[1], U.shape[0], factor, _ptr(U), U.shape[1], _ptr(O), O.shape[1], _ptr(M),
                        M.shape[1])


def matmul(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    C_ = np.zeros((A.shape[0], B.shape[1]))
    lib().oracle_matmul(A.shape[0], B.shape[1], A.shape[1], _ptr(A), A.shape[1], _ptr(B), B.shape[1], _ptr(C_),
                        B.shape[1])
    return C_


def prod_fit(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """c++/numerics.hpp:283-306."""
    if B.shape[0] <= A.shape[1]:
        if A.shape[0] == 0 or B.shape[1] == 0:
            return np.zeros((0, 0))
        return matmul(np.ascontiguousarray(A[:, :B.shape[0]]), B)
    if A.shape[0] == 0 or B.shape[1] == 0:
        return np.zeros((0, 0))
    return matmul(A, np.ascontiguousarray(B[:A.shape[1], :]))


def chit_weight(En: float, Em: float, beta: float) -> float:
    return lib().oracle_chit_weight(En, Em, beta)


class ChainBinning:
    """Bins pair (positive/negative energies) of c++/spectrum.hpp:12-31 on the standard
    log grid of c++/bins.hpp:61-100; weights are complex (re, im arrays)."""

    def __init__(self, log10emin: float, log10emax: float, bins: int, discard_immediately: float = 0.0):
        self.log10emin, self.bins, self.discard = float(log10emin), int(bins), float(discard_immediately)
        self.nbins = lib().oracle_loggrid(log10emin, log10emax, bins, None)
        self.energies = np.zeros(self.nbins)
        lib().oracle_loggrid(log10emin, log10emax, bins, _ptr(self.energies))
        self.pos_re, self.pos_im = np.zeros(self.nbins), np.zeros(self.nbins)
        self.neg_re, self.neg_im = np.zeros(self.nbins), np.zeros(self.nbins)

    def _arrs(self):
        return _ptr(self.pos_re), _ptr(self.pos_im), _ptr(self.neg_re), _ptr(self.neg_im)

    def add(self, energy: np.ndarray, weight_re: np.ndarray, factor: float = 1.0, weight_im=None) -> None:
        e = np.ascontiguousarray(energy, dtype=np.float64)
        wr = np.ascontiguousarray(weight_re, dtype=np.float64)
        wi = None if weight_im is None else np.ascontiguousarray(weight_im, dtype=np.float64)
        lib().oracle_chain_add(*self._arrs(), self.nbins, self.log10emin, self.bins, self.discard, e.size, _ptr(e),
                               _ptr(wr), None if wi is None else _ptr(wi), factor)

    def dmnrg_pair(self, Em, Ej, op1, op2, rhoP, rho1, factor, sign, Emin, Emax):
        """Algo_DMNRG::calc inner loops (c++/algo_DMNRG.hpp:29-52) for one pair."""
        kp, k1 = len(Em), len(Ej)
        Em = np.ascontiguousarray(Em, dtype=np.float64)
        Ej = np.ascontiguousarray(Ej, dtype=np.float64)
        op1, op2 = np.ascontiguousarray(op1), np.ascontiguousarray(op2)
        rhoP, rho1 = np.ascontiguousarray(rhoP), np.ascontiguousarray(rho1)
        lib().oracle_dmnrg_pair(kp, k1, _ptr(Em), _ptr(Ej), _ptr(op1), op1.shape[1], _ptr(op2), op2.shape[1],
                                _ptr(rhoP), rhoP.shape[1], _ptr(rho1), rho1.shape[1], factor, sign, Emin, Emax,
                                *self._arrs(), self.nbins, self.log10emin, self.bins, self.discard)

    def fdm_pair(self, which: str, Ei, Ki, Ej, Kj, op1, op2, rho, factor, sign, T, wnf):
        """Algo_FDMgt/ls::calc (c++/algo_FDM.hpp:84-114 / 30-60) for one pair."""
        Ei = np.ascontiguousarray(Ei, dtype=np.float64)
        Ej = np.ascontiguousarray(Ej, dtype=np.float64)
        op1, op2, rho = np.ascontiguousarray(op1), np.ascontiguousarray(op2), np.ascontiguousarray(rho)
        rd = rho.shape[0]
        lib().oracle_fdm_pair(0 if which == "gt" else 1, len(Ei), Ki, len(Ej), Kj, _ptr(Ei), _ptr(Ej), _ptr(op1),
                              op1.shape[1], _ptr(op2), op2.shape[1], _ptr(rho), max(rd, 1), rd, factor, sign, T, wnf,
                              *self._arrs(), self.nbins, self.log10emin, self.bins, self.discard)


def windowfunction(E, Emin, Ex, Emax, last=False, first=False, zbw=False, NNtanh=0.0) -> float:
    flags = (1 if last else 0) | (2 if first else 0) | (4 if zbw else 0)
    return lib().oracle_windowfunction(E, Emin, Ex, Emax, flags, NNtanh)
