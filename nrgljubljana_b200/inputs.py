"""Readers for NRG Ljubljana's run inputs: the ``param`` file and the ``data`` file.

``data`` (format version 9) is what the reference's initialisation tool writes and what
``InputData`` reads (c++/read-input.hpp:23-134): a header of ``#`` lines carrying the
version (``#!9``) and the symmetry type, the numbers of channels, chain sites and
subspaces, the initial subspaces with their energies (c++/eigen.hpp:307-317), the
<||f||> matrices per channel (c++/operators.hpp:142-155), then lettered blocks: ``e``
ground-state energy, ``s``/``p``/``g``/``d``/``t``/``o``/``q`` operator matrices
(c++/operators.hpp:30-41) and ``z`` the Wilson-chain tables xi and zeta
(c++/coef.hpp:21-52). Host-side parsing only.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

Invar = Tuple[int, ...]
Pair = Tuple[Invar, Invar]

DATA_VERSION = 9


def parse_param(text: str) -> Dict[str, str]:
    """key=value lines of a ``param`` file; ``[section]`` and ``#`` lines are skipped."""
    out: Dict[str, str] = {}
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("#") or line.startswith("["):
            continue
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        out[k.strip()] = v.strip()
    return out


@dataclass
class DataFile:
    symtype: str
    channels: int
    nmax: int
    subspaces: List[Tuple[Invar, np.ndarray]]          # initial subspaces in file order
    opch: List[List[Dict[Pair, np.ndarray]]]           # [channel][perchannel] -> <I1||f||I2>
    gs_energy: float = 0.0
    ops: Dict[str, Tuple[str, Dict[Pair, np.ndarray]]] = field(default_factory=dict)  # name -> (kind, matrices)
    xi: List[np.ndarray] = field(default_factory=list)   # per coefficient channel, index 0..Nmax
    zeta: List[np.ndarray] = field(default_factory=list)


class _Lines:
    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.i = 0
        self.tok: List[str] = []

    def _fill(self) -> bool:
        while not self.tok:
            if self.i >= len(self.lines):
                return False
            line = self.lines[self.i]
            self.i += 1
            if line.lstrip().startswith("#"):
                continue
            self.tok = line.split()
        return True

    def word(self) -> str:
        if not self._fill():
            raise ValueError("data file ended early")
        return self.tok.pop(0)

    def int(self) -> int:
        return int(self.word())

    def float(self) -> float:
        return float(self.word())

    def block(self):
        """Next lettered block: (letter, rest of the line) or None at the end."""
        if self.tok:
            raise ValueError("unread values before a block marker")
        while self.i < len(self.lines):
            line = self.lines[self.i].strip()
            self.i += 1
            if not line:
                continue
            if line.startswith("#"):
                continue
            return line[0], line[1:].strip()
        return None


def _invar(L: _Lines, dim: int) -> Invar:
    return tuple(L.int() for _ in range(dim))


def _matrix_elements(L: _Lines, dims: Dict[Invar, int], invdim: int) -> Dict[Pair, np.ndarray]:
    nf = L.int()
    out: Dict[Pair, np.ndarray] = {}
    for _ in range(nf):
        I1 = _invar(L, invdim)
        I2 = _invar(L, invdim)
        if I1 not in dims or I2 not in dims:
            raise ValueError("Corrupted input file.")
        r, c = dims[I1], dims[I2]
        out[(I1, I2)] = np.array([L.float() for _ in range(r * c)], dtype=np.float64).reshape(r, c)
    return out


INVDIM = {"QS": 2}


def read_data(text: str, perchannel: int = 1) -> DataFile:
    lines = text.splitlines()
    version = -1
    symtype = ""
    k = 0
    while k < len(lines) and lines[k].startswith("#"):
        line = lines[k]
        if line.startswith("#!"):
            version = int(line[2:].split()[0])
        elif "symtype" in line[1:]:
            symtype = line.replace("\t", " ").rstrip().rsplit(" ", 1)[-1]
        k += 1
    if version != DATA_VERSION:
        raise ValueError(f"data file version {version}, expected {DATA_VERSION}")
    if symtype not in INVDIM:
        raise ValueError(f"symtype {symtype!r} is not supported")
    invdim = INVDIM[symtype]
    L = _Lines("\n".join(lines[k:]))
    channels, nmax, nsubs = L.int(), L.int(), L.int()
    subs: List[Tuple[Invar, np.ndarray]] = []
    for _ in range(nsubs):
        I = _invar(L, invdim)
        n = L.int()
        subs.append((I, np.array([L.float() for _ in range(n)], dtype=np.float64)))
    dims = {I: len(e) for I, e in subs}
    opch: List[List[Dict[Pair, np.ndarray]]] = []
    for _ in range(channels):
        per = []
        for _ in range(perchannel):
            blk = L.block()
            if blk is None or blk[0] != "f":
                raise ValueError("expected an 'f' block")
            per.append(_matrix_elements(L, dims, invdim))
        opch.append(per)
    d = DataFile(symtype, channels, nmax, subs, opch)
    while True:
        blk = L.block()
        if blk is None:
            break
        ch, name = blk
        if ch == "e":
            d.gs_energy = L.float()
        elif ch in "spgdtoq":
            d.ops[name] = (ch, _matrix_elements(L, dims, invdim))
        elif ch == "z":
            for tab in (d.xi, d.zeta):
                for _ in range(channels):
                    nr = L.int()
                    tab.append(np.array([L.float() for _ in range(nr + 1)], dtype=np.float64))
        else:
            raise ValueError(f"Unknown block {ch} in data file.")
    if not d.xi or len(d.xi[0]) - 1 != nmax:
        raise ValueError("length of the coefficient table differs from Nmax")
    return d


def SCALE(N: int, Lambda: float, discretization: str = "Z", z: float = 1.0, bandrescale: float = 1.0) -> float:
    """Energy scale of the length-N chain (c++/params.hpp:619-634, no substeps)."""
    scale = 0.0
    if discretization == "Y":
        scale = 0.5 * (1.0 + 1.0 / Lambda)
    if discretization in ("C", "Z"):
        scale = (1.0 - 1.0 / Lambda) / math.log(Lambda)
    scale *= Lambda ** (-(N - 1) / 2.0 + 1 - z)
    if scale == 0.0:
        raise ValueError(f"unsupported discretization {discretization!r}")
    return scale * bandrescale
