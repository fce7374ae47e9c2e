"""ctypes binding of the C-ABI in include/nrg_b200.h (libnrg_b200.so).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnrg_b200.so")

NRG_OK = 0
NRG_ERR_ARG = -1
NRG_ERR_CUDA = -2
NRG_ERR_OOM = -3
NRG_ERR_NODEV = -4
NRG_DIAG_MAX_N = 10240

NRG_SPEC_DMNRG = 0
NRG_SPEC_FDMGT = 1
NRG_SPEC_FDMLS = 2
NRG_SPEC_FDMMATS = 3
NRG_SPEC_FTMATS = 4

# Every symbol include/nrg_b200.h declares.
EXPORTS = ("nrg_version", "nrg_last_error", "nrg_create", "nrg_destroy", "nrg_trim", "nrg_diag_batch",
           "nrg_diag_batch_host",
           "nrg_gemm3_batch", "nrg_gemm3_batch_host", "nrg_transform_noalloc", "nrg_spec_accumulate",
           "nrg_spec_accumulate_mats", "nrg_profile",
           "nrg_profile_read", "nrg_bins_grid", "nrg_hamiltonian_batch",
           "nrg_broaden", "nrg_get_tuning", "nrg_set_tuning")
NRG_NOALLOC_SCRATCH_DOUBLES = 1 << 20


class Gemm3(C.Structure):
    _fields_ = [("M", C.c_void_p), ("ldm", C.c_int64), ("A", C.c_void_p), ("lda", C.c_int64),
                ("O", C.c_void_p), ("ldo", C.c_int64), ("B", C.c_void_p), ("ldb", C.c_int64),
                ("rows", C.c_int), ("cols", C.c_int), ("ka", C.c_int), ("kb", C.c_int),
                ("transA", C.c_int), ("transB", C.c_int), ("factor", C.c_double)]


NRG_HP_DIAG = 0
NRG_HP_BLOCK = 1


class HPiece(C.Structure):
    _fields_ = [("blk", C.c_int), ("kind", C.c_int), ("r0", C.c_int), ("c0", C.c_int), ("rows", C.c_int),
                ("cols", C.c_int), ("trans", C.c_int), ("pad_", C.c_int), ("ld", C.c_int64), ("src", C.c_void_p),
                ("factor", C.c_double), ("shift", C.c_double)]


def _np_layout(struct) -> "np.dtype":
    """numpy record type with the byte layout of a ctypes Structure, for descriptor arrays
    built vectorised on the host and handed to the library as one pointer."""
    import numpy as np
    kinds = {C.c_void_p: "u8", C.c_int64: "i8", C.c_int: "i4", C.c_double: "f8"}
    names = [f[0] for f in struct._fields_]
    return np.dtype({"names": names, "formats": [kinds[f[1]] for f in struct._fields_],
                     "offsets": [getattr(struct, n).offset for n in names], "itemsize": C.sizeof(struct)})


GEMM3_DTYPE = _np_layout(Gemm3)
HPIECE_DTYPE = _np_layout(HPiece)


class SpecPair(C.Structure):
    _fields_ = [("Ei", C.c_void_p), ("Ej", C.c_void_p), ("op1", C.c_void_p), ("ld1", C.c_int64),
                ("op2", C.c_void_p), ("ld2", C.c_int64), ("rho_i", C.c_void_p), ("ldri", C.c_int64),
                ("rho_j", C.c_void_p), ("ldrj", C.c_int64), ("ni", C.c_int), ("ki", C.c_int),
                ("nj", C.c_int), ("kj", C.c_int), ("rdi", C.c_int), ("rdj", C.c_int), ("factor", C.c_double)]


SPECPAIR_DTYPE = _np_layout(SpecPair)


class SpecParams(C.Structure):
    _fields_ = [("algo", C.c_int), ("sign", C.c_int), ("T", C.c_double), ("wnf", C.c_double),
                ("Emin", C.c_double), ("Emax", C.c_double)]


class Bins(C.Structure):
    _fields_ = [("log10emin", C.c_double), ("log10emax", C.c_double), ("bins", C.c_int), ("nbins", C.c_int),
                ("discard_immediately", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("small_max_n", C.c_int), ("mid_max_n", C.c_int), ("cluster_max_n", C.c_int),
                ("reduction_ctas_per_sm", C.c_int), ("band_min_n", C.c_int), ("band_max_blocks", C.c_int)]


class PhaseStat(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("ms", C.c_double), ("launches", C.c_longlong)]


_lib = None


def load() -> C.CDLL:
    """Load libnrg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with nrgljubljana_b200.build.build() "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    L.nrg_version.restype = C.c_int
    L.nrg_last_error.restype = C.c_char_p
    L.nrg_create.argtypes = [C.POINTER(P), C.c_int, C.c_size_t]
    L.nrg_destroy.argtypes = [P]
    L.nrg_trim.argtypes = [P]
    L.nrg_diag_batch.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(P), C.POINTER(P), C.POINTER(P),
                                 C.POINTER(C.c_int), P]
    L.nrg_diag_batch_host.argtypes = L.nrg_diag_batch.argtypes
    L.nrg_gemm3_batch.argtypes = [P, C.c_int, C.POINTER(Gemm3), P]
    L.nrg_gemm3_batch_host.argtypes = L.nrg_gemm3_batch.argtypes
    L.nrg_spec_accumulate.argtypes = [P, C.c_int, C.POINTER(SpecPair), C.POINTER(SpecParams), C.POINTER(Bins), P, P, P]
    L.nrg_spec_accumulate_mats.argtypes = [P, C.c_int, C.POINTER(SpecPair), C.POINTER(SpecParams), C.c_int, P, P, P]
    L.nrg_bins_grid.argtypes = [C.POINTER(Bins), C.POINTER(C.c_double)]
    L.nrg_transform_noalloc.argtypes = [P, C.c_int64, P, C.c_int64, P, C.c_int64, P, C.c_int64, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.c_double, P]
    L.nrg_hamiltonian_batch.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.POINTER(P), C.c_int, C.POINTER(HPiece), P]
    L.nrg_broaden.argtypes = [P, C.c_int, P, P, C.c_int, P, C.c_double, C.c_double, P, P]
    L.nrg_get_tuning.argtypes = [P, C.POINTER(Tuning)]
    L.nrg_set_tuning.argtypes = [P, C.POINTER(Tuning)]
    L.nrg_profile.argtypes = [P, C.c_int]
    L.nrg_profile_read.argtypes = [P, C.POINTER(PhaseStat), C.c_int]
    _lib = L
    return L


def last_error() -> str:
    return load().nrg_last_error().decode()


class NRGError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where} failed with code {code}: {last_error()}")
        self.code = code


def check(code: int, where: str) -> int:
    if code < 0:
        raise NRGError(code, where)
    return code
