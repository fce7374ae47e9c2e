"""Symmetry type QS (charge Q, total spin SS = 2S+1), one channel, without substeps.

The tables below are the reference's coefficient tables for this symmetry, restated:
  In / QN                c++/symmetry/coefnew/qs/qs-1ch-In2.dat, qs-1ch-QN.dat
  diagonal shifts        c++/symmetry/coefnew/qs/qs-1ch-diag.dat
  off-diagonal factors   c++/symmetry/coefnew/qs/qs-1ch-offdiag.dat
  <||f||> recalculation  c++/symmetry/coefnew/qs/qs-1ch-spinupa.dat, qs-1ch-spindowna.dat
                         (driven by SymmetryQS::recalc_irreduc, c++/symmetry/nrg-recalc-QS.hpp:192-330)
and the rules of c++/symmetry/sym-QS-impl.hpp:13-93 and c++/symmetry.hpp:31-35, 87-113.
A factor is evaluated only when its block contributes, as the reference's macros do, so
that no factor with a division by zero is ever formed.
"""
from __future__ import annotations

import math
from typing import Callable, List, Tuple

Invar = Tuple[int, int]

COMBS = 4
# In[i]: the ancestor of subspace I through combination i is I + In[i] (c++/symmetry.hpp:100-105).
IN: List[Invar] = [(1, 0), (0, -1), (0, 1), (-1, 0)]
# QN[i]: quantum numbers of the added site's states in combination i.
QN: List[Invar] = [(-1, 1), (0, 2), (0, 2), (1, 1)]


def S(ss: int) -> float:
    """Spin from multiplicity (c++/invar.hpp:22)."""
    return (ss - 1.0) / 2.0


def mult(I: Invar) -> int:
    return I[1]


def allowed(I: Invar) -> bool:
    return I[1] > 0


def su2_triangle(ss1: int, ss2: int, ss3: int) -> bool:
    return abs(ss1 - ss2) <= ss3 - 1 and abs(ss2 - ss3) <= ss1 - 1 and abs(ss3 - ss1) <= ss2 - 1


def triangle(I1: Invar, I2: Invar, I3: Invar) -> bool:
    return I1[0] == I2[0] + I3[0] and su2_triangle(I1[1], I2[1], I3[1])


def ancestors(I: Invar) -> List[Invar]:
    return [(I[0] + d[0], I[1] + d[1]) for d in IN]


def new_subspaces(I: Invar) -> List[Invar]:
    return [(I[0] - d[0], I[1] - d[1]) for d in IN]


# (i, j, channel, factor(ss)) with 1-based combination indexes; the block (i, j) gets
# factor * xi(N, ch) / scale * <In[i]||f||In[j]>.
OFFDIAG: List[Tuple[int, int, int, Callable[[int], float]]] = [
    (1, 2, 0, lambda ss: 1.0),
    (1, 3, 0, lambda ss: 1.0),
    (2, 4, 0, lambda ss: -(math.sqrt(2) * math.sqrt(S(ss) / (1 + 2 * S(ss))))),
    (3, 4, 0, lambda ss: (1 + S(ss)) / math.sqrt(0.5 + (3 * S(ss)) / 2. + S(ss) ** 2)),
]

# (i, channel, number of electrons added): the diagonal of block i gets
# zeta(N+1, ch) * (number - avgoccup) / scale, avgoccup = 1 for spin-1/2 electrons.
DIAG: List[Tuple[int, int, float]] = [(1, 0, 0.0), (2, 0, 1.0), (3, 0, 1.0), (4, 0, 2.0)]
AVGOCCUP = 1.0

# <I1||f||Ip> for I1 = Ip + (1, +1) and I1 = Ip + (1, -1): rows (i1, ip, factor(ssp)).
RECALC_F: List[Tuple[Invar, List[Tuple[int, int, Callable[[int], float]]]]] = [
    ((1, 1), [(2, 1, lambda ssp: 1.0),
              (4, 3, lambda ssp: -math.sqrt(1 - 1 / (2. * (1 + S(ssp)))))]),
    ((1, -1), [(3, 1, lambda ssp: 1.0),
               (4, 2, lambda ssp: math.sqrt(1 + 1 / (2. * S(ssp))))]),
]

TD_FIELDS = ("<Sz^2>", "<Q>", "<Q^2>")


def td_extra(Zs, subspaces, Z: float) -> List[float]:
    """<Sz^2>, <Q>, <Q^2> of SymmetryQS::calculate_TD (c++/symmetry/sym-QS-impl.hpp:72-86);
    Zs[k] is the multiplicity-weighted Boltzmann sum of subspaces[k]."""
    trSZ = trQ = trQ2 = 0.0
    for sumZ, (q, ss) in zip(Zs, subspaces):
        trQ += sumZ * q
        trQ2 += sumZ * q * q
        trSZ += sumZ * (ss * ss - 1) / 12.
    return [trSZ / Z, trQ / Z, trQ2 / Z]

# Doublet operators <I1||O||Ip> with Ip = I1 + (-1, +1) (qs-1ch-doubletp.dat) and
# Ip = I1 + (-1, -1) (qs-1ch-doubletm.dat), driven by SymmetryQS::recalc_doublet
# (c++/symmetry/nrg-recalc-QS.hpp:32-117): rows (i1, ip, factor(ss1)); the old matrix is the
# one between the ancestors of I1 through i1 and of Ip through ip.
DOUBLET: List[Tuple[Invar, List[Tuple[int, int, Callable[[int], float]]]]] = [
    ((-1, 1), [(1, 1, lambda ss: 1.0),
               (2, 2, lambda ss: (-2 * math.sqrt(S(ss) * (1 + S(ss)))) / (1 + 2 * S(ss))),
               (3, 2, lambda ss: 1 / (1 + 2 * S(ss))),
               (3, 3, lambda ss: -1.0),
               (4, 4, lambda ss: 1.0)]),
    ((-1, -1), [(1, 1, lambda ss: 1.0),
                (2, 2, lambda ss: -1.0),
                (2, 3, lambda ss: 1 / (-1 - 2 * S(ss))),
                (3, 3, lambda ss: (-2 * (1 + S(ss))) / math.sqrt(5 + 1 / S(ss) + 8 * S(ss) + 4 * S(ss) ** 2)),
                (4, 4, lambda ss: 1.0)]),
]


def specdens_factor(Ip: Invar, I1: Invar) -> float:
    """SymmetryQS::specdens_factor (c++/symmetry/sym-QS-impl.hpp:64-70)."""
    return S(Ip[1]) + 1.0 if I1[1] == Ip[1] + 1 else S(Ip[1])
