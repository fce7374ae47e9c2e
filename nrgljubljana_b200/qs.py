"""Symmetry type QS (charge Q, total spin SS = 2S+1), one or two channels, without substeps.

The tables below are the reference's coefficient tables for this symmetry, restated:
  In / QN                c++/symmetry/coefnew/qs/qs-{1,2}ch-In2.dat, qs-{1,2}ch-QN.dat
  diagonal shifts        c++/symmetry/coefnew/qs/qs-{1,2}ch-diag.dat
  off-diagonal factors   c++/symmetry/coefnew/qs/qs-{1,2}ch-offdiag.dat
  <||f||> recalculation  c++/symmetry/coefnew/qs/qs-1ch-spin{up,down}a.dat,
                         qs-2ch-spin{up,down}{a,b}.dat (channel 0: a, channel 1: b)
                         (driven by SymmetryQS::recalc_irreduc, c++/symmetry/nrg-recalc-QS.hpp:192-460)
  doublet recalculation  c++/symmetry/coefnew/qs/qs-{1,2}ch-doublet{p,m}.dat
                         (SymmetryQS::recalc_doublet, c++/symmetry/nrg-recalc-QS.hpp:32-117)
  triplet recalculation  c++/symmetry/coefnew/qs/qs-{1,2}ch-triplet{s,p,m}.dat
                         (SymmetryQS::recalc_triplet, c++/symmetry/nrg-recalc-QS.hpp:495-640)
and the rules of c++/symmetry/sym-QS-impl.hpp:13-93 and c++/symmetry.hpp:31-35, 87-113.
A factor is evaluated only when its blocks are not empty, as the reference's macros and
the empty-block checks of product/transform arrange, so that no factor with a division by
zero (S = 0) is ever used. The triplet factors are evaluated in IEEE double arithmetic, as
the reference's C++ evaluates them: 1/sqrt(x/0) is 0, and a row whose factor is not finite is
an error when it is used.
"""
from __future__ import annotations

import math
from typing import Callable, Dict, List, Tuple

import numpy as np

Invar = Tuple[int, int]
Fn = Callable[[int], float]


def S(ss: int) -> np.float64:
    """Spin from multiplicity (c++/invar.hpp:22), as a numpy double so that the table factors
    divide by zero as the reference's C++ does (see ieee)."""
    return np.float64((ss - 1.0) / 2.0)


_IEEE_CACHE: dict = {}


def ieee(fn, ss: int) -> float:
    """A table factor at SS = ss, evaluated as the reference's C++ evaluates it: in IEEE double
    arithmetic, x/0 is +-inf and the square root of a negative number is nan (the rows where
    that happens are never used, but a factor at S = 0 may still come out finite, e.g.
    1/sqrt(2 + 2/S) = 0). The factors are pure functions of (row, SS): each is evaluated
    once per process and then looked up (a run asks for the same few thousand every step)."""
    key = (fn, ss)
    v = _IEEE_CACHE.get(key)
    if v is None:
        with np.errstate(all="ignore"):
            try:
                v = float(fn(ss))
            except ValueError:  # math.sqrt of a negative number
                v = math.nan
        _IEEE_CACHE[key] = v
    return v


def mult(I: Invar) -> int:
    return I[1]


def allowed(I: Invar) -> bool:
    return I[1] > 0


def su2_triangle(ss1: int, ss2: int, ss3: int) -> bool:
    return abs(ss1 - ss2) <= ss3 - 1 and abs(ss2 - ss3) <= ss1 - 1 and abs(ss3 - ss1) <= ss2 - 1


def triangle(I1: Invar, I2: Invar, I3: Invar) -> bool:
    return I1[0] == I2[0] + I3[0] and su2_triangle(I1[1], I2[1], I3[1])


AVGOCCUP = 1.0  # per channel: multiplicity 2 of an electron divided by 2
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


def specdens_factor(Ip: Invar, I1: Invar) -> float:
    """SymmetryQS::specdens_factor (c++/symmetry/sym-QS-impl.hpp:64-70)."""
    return S(Ip[1]) + 1.0 if I1[1] == Ip[1] + 1 else S(Ip[1])


def dynamicsusceptibility_factor(Ip: Invar, I1: Invar) -> float:
    """SymmetryQS::dynamicsusceptibility_factor (c++/symmetry/sym-QS-impl.hpp:56-62)."""
    ssp, ss1 = Ip[1], I1[1]
    if ss1 == ssp + 2:
        return 1.0 + (ssp - 1) / 3.0
    if ss1 == ssp:
        return ssp / 3.0
    if ss1 == ssp - 2:
        return (ssp - 2) / 3.0
    raise AssertionError("abs(ss1 - ssp) == 2 || ss1 == ssp")


def correlator_factor(Ip: Invar, I1: Invar) -> float:
    """CorrelatorFactorFnc (c++/symmetry.hpp:235): the multiplicity of I1."""
    return float(mult(I1))


_TRIPLET_CACHE: dict = {}


def triplet_factor(fn, ss1: int) -> float:
    """A triplet-table factor at SS = ss1 in IEEE double arithmetic (evaluated once per
    (row, SS) per process, as ieee)."""
    key = (fn, ss1)
    v = _TRIPLET_CACHE.get(key)
    if v is None:
        with np.errstate(all="ignore"):
            v = float(fn(np.float64((ss1 - 1) / 2.0)))
        _TRIPLET_CACHE[key] = v
    if not math.isfinite(v):
        raise AssertionError(f"triplet recalculation factor is not finite at SS={ss1}")
    return v


class Tables:
    """The coefficient tables of one channel count.

    IN[i]       the ancestor of subspace I through combination i is I + IN[i]
    QN[i]       quantum numbers of the added shell's states of combination i
    OFFDIAG     (i, j, channel, factor(ss)), 1-based combinations: block (i, j) gets
                factor * xi(N, ch) / scale * <IN[i]||f_ch||IN[j]>
    DIAG        (i, channel, electrons added in that channel): the diagonal of block i gets
                zeta(N+1, ch) * (number - AVGOCCUP) / scale
    DIAG_FIRST  whether make_matrix lists the diagonal table before the off-diagonal one
    RECALC_F    (dq, channel, rows (i1, ip, factor(ssp))): <I1||f_ch||Ip> for I1 = Ip + dq
    DOUBLET     (dq, rows (i1, ip, factor)): a doublet operator for Ip = I1 + dq; the factor is
                evaluated by doublet_factor(fn, ss1)
    TRIPLET     (dq, rows (i1, ip, factor(S1))): a triplet operator for Ip = I1 + dq, the factor
                a function of the spin S1 of I1 (a numpy float64), see triplet_factor
    GLOBAL      name -> rows (i1, ip, channel, value) of the global charge operators
                (SymmetryQS::recalc_global, c++/symmetry/nrg-recalc-QS.hpp:680-740): after the
                singlet recalculation, <I||Q||I> += value * U_i1 U_ip^T for every subspace I
    """

    def __init__(self, channels, IN, QN, OFFDIAG, DIAG, DIAG_FIRST, RECALC_F, DOUBLET, TRIPLET,
                 doublet_of_spin=False):
        self.channels = channels
        self.COMBS = len(IN)
        self.IN, self.QN = IN, QN
        self.OFFDIAG, self.DIAG, self.DIAG_FIRST = OFFDIAG, DIAG, DIAG_FIRST
        self.RECALC_F, self.DOUBLET, self.TRIPLET = RECALC_F, DOUBLET, TRIPLET
        self._doublet_of_spin = doublet_of_spin
        self.GLOBAL = global_charges(DIAG) if channels == 2 else {}

    def doublet_factor(self, fn, ss1: int) -> float:
        """A doublet-table factor at SS = ss1 (rows of the two-channel tables are functions of
        the spin, evaluated as the triplet rows are)."""
        return triplet_factor(fn, ss1) if self._doublet_of_spin else ieee(fn, ss1)

    def ancestors(self, I: Invar) -> List[Invar]:
        return [(I[0] + d[0], I[1] + d[1]) for d in self.IN]

    def new_subspaces(self, I: Invar) -> List[Invar]:
        return [(I[0] - d[0], I[1] - d[1]) for d in self.IN]


def global_charges(diag) -> Dict[str, List[Tuple[int, int, int, int]]]:
    """The global operators of two-channel QS: the charge the new site adds in channel 0 (Q1)
    and in channel 1 (Q2), their difference Q2 - Q1 (Qdiff) and the total charge counted
    from half filling, sum over the channels of (n_ch - 1) (Qtot). A combination i that adds
    n electrons in channel ch contributes the row (i, i, ch, value) where value is nonzero,
    channel 0 rows first, by combination (the reference's qs-2ch-{q1,q2,qdiff,qtot}.dat)."""
    n = {(i, ch): int(num) for i, ch, num in diag}
    combs = sorted({i for i, _ in n})
    rows = {"Q1": [(i, i, 0, n[i, 0]) for i in combs],
            "Q2": [(i, i, 1, n[i, 1]) for i in combs],
            "Qdiff": [(i, i, 0, -n[i, 0]) for i in combs] + [(i, i, 1, n[i, 1]) for i in combs],
            "Qtot": [(i, i, ch, n[i, ch] - 1) for ch in (0, 1) for i in combs]}
    return {name: [r for r in rs if r[3] != 0] for name, rs in rows.items()}


def _one(ss):
    return 1.0


QS1 = Tables(
    1,
    IN=[(1, 0), (0, -1), (0, 1), (-1, 0)],
    QN=[(-1, 1), (0, 2), (0, 2), (1, 1)],
    OFFDIAG=[
        (1, 2, 0, _one),
        (1, 3, 0, _one),
        (2, 4, 0, lambda ss: -(math.sqrt(2) * math.sqrt(S(ss) / (1 + 2 * S(ss))))),
        (3, 4, 0, lambda ss: (1 + S(ss)) / math.sqrt(0.5 + (3 * S(ss)) / 2. + S(ss) ** 2)),
    ],
    DIAG=[(1, 0, 0.0), (2, 0, 1.0), (3, 0, 1.0), (4, 0, 2.0)],
    DIAG_FIRST=False,
    RECALC_F=[
        ((1, 1), 0, [(2, 1, _one), (4, 3, lambda ssp: -math.sqrt(1 - 1 / (2. * (1 + S(ssp)))))]),
        ((1, -1), 0, [(3, 1, _one), (4, 2, lambda ssp: math.sqrt(1 + 1 / (2. * S(ssp))))]),
    ],
    DOUBLET=[
        ((-1, 1), [(1, 1, _one),
                   (2, 2, lambda ss: (-2 * math.sqrt(S(ss) * (1 + S(ss)))) / (1 + 2 * S(ss))),
                   (3, 2, lambda ss: 1 / (1 + 2 * S(ss))),
                   (3, 3, lambda ss: -1.0),
                   (4, 4, _one)]),
        ((-1, -1), [(1, 1, _one),
                    (2, 2, lambda ss: -1.0),
                    (2, 3, lambda ss: 1 / (-1 - 2 * S(ss))),
                    (3, 3, lambda ss: (-2 * (1 + S(ss))) / math.sqrt(5 + 1 / S(ss) + 8 * S(ss) + 4 * S(ss) ** 2)),
                    (4, 4, _one)]),
    ],
    TRIPLET=[
        ((0, 0), [(1, 1, lambda s: 1.0),
                  (2, 2, lambda s: np.sqrt(1 - 1 / s + 2 / (1 + 2 * s))),
                  (2, 3, lambda s: 1 / np.sqrt((1 + s) * (1 + 2 * s))),
                  (3, 2, lambda s: -(1 / np.sqrt(s * (1 + 2 * s)))),
                  (3, 3, lambda s: (1 + s) * np.sqrt((s * (1 + 2 * s)) / ((1 + s) ** 3 * (3 + 2 * s)))
                   + 2 * np.sqrt(s / (3 + 11 * s + 12 * s ** 2 + 4 * s ** 3))),
                  (4, 4, lambda s: 1.0)]),
        ((0, 2), [(1, 1, lambda s: 1.0),
                  (2, 2, lambda s: np.sqrt(1 + 1 / (1 + s) - 2 / (1 + 2 * s))),
                  (3, 2, lambda s: -(1 / np.sqrt((1 + s) * (1 + 2 * s)))),
                  (3, 3, lambda s: 1.0),
                  (4, 4, lambda s: 1.0)]),
        ((0, -2), [(1, 1, lambda s: 1.0),
                   (2, 2, lambda s: 1.0),
                   (2, 3, lambda s: 1 / np.sqrt(s * (1 + 2 * s))),
                   (3, 3, lambda s: (np.sqrt((-1 + 4 * s ** 2) / (s + s ** 2))
                                     + np.sqrt((-1 + 2 * s) / (s + 3 * s ** 2 + 2 * s ** 3))) / 2.),
                   (4, 4, lambda s: 1.0)]),
    ],
)


def _a(ss):  # sqrt(S/(1+2S))
    return math.sqrt(S(ss) / (1 + 2 * S(ss)))


def _b(ss):  # (1+S)/sqrt((1+S)(1+2S))
    return (1 + S(ss)) / math.sqrt((1 + S(ss)) * (1 + 2 * S(ss)))


def _b2(ss):  # sqrt(2)(1+S)/sqrt((1+S)(1+2S))
    return (math.sqrt(2) * (1 + S(ss))) / math.sqrt((1 + S(ss)) * (1 + 2 * S(ss)))


def _c(ssp):  # 1/sqrt(1 + 1/(1+2S))
    return 1 / math.sqrt(1 + 1 / (1 + 2 * S(ssp)))


# two-channel triplet rows (qs-2ch-triplet{s,p,m}.dat); combinations 2/4, 3/5, 12/14 and
# 13/15 carry the same factors
def _t_lo(s):   # (i, i) for the lower-spin ancestor of a doublet shell
    return 1 / np.sqrt((s * (1 + 2 * s)) / (-1 + s + 2 * s ** 2))


def _t_x(s):    # lower -> higher
    return 1 / np.sqrt((1 + s) * (1 + 2 * s))


def _t_y(s):    # higher -> lower
    return -(1 / np.sqrt(s * (1 + 2 * s)))


def _t_hi(s):   # (i, i) for the higher-spin ancestor
    return (3 + 2 * s) / np.sqrt(((1 + s) * (3 + 4 * s * (2 + s))) / s)


def _t_1111(s):
    r = (s * (2 + s) * (1 + 2 * s) ** 2) / ((1 + s) * (3 + 2 * s) ** 2)
    a = s * (1 + s) * (2 + s)
    num = (12 * np.sqrt(a) + 33 * np.sqrt(s ** 4 * a) + 24 * np.sqrt(s ** 6 * a) + 4 * np.sqrt(s ** 8 * a)
           + 18 * np.sqrt(r) + s * (29 * np.sqrt(a) + 60 * np.sqrt(r) + 2 * s * np.sqrt(r) * (31 + 10 * s)))
    return num / ((1 + s) ** 2.5 * (2 + s) * (3 + 2 * s) ** 2)


def _u(s):      # 1.0 whatever s
    return 1.0


_T2S = ([(1, 1, _u)]
        + [r for a, b in ((2, 3), (4, 5)) for r in ((a, a, _t_lo), (a, b, _t_x), (b, a, _t_y), (b, b, _t_hi))]
        + [(6, 6, _u), (7, 7, _u), (8, 8, _u),
           (9, 9, lambda s: np.sqrt(-1 + s ** 2) / s),
           (9, 10, lambda s: np.sqrt(1 - 2 / (1 + 2 * s)) / s),
           (10, 9, lambda s: -(1 / s)),
           (10, 10, lambda s: 1 - 1 / s + 1 / (1 + s)),
           (10, 11, lambda s: 1 / (1 + s)),
           (11, 10, lambda s: -((3 + 2 * s) / ((1 + s) * np.sqrt(3 + 4 * s * (2 + s))))),
           (11, 11, _t_1111)]
        + [r for a, b in ((12, 13), (14, 15)) for r in ((a, a, _t_lo), (a, b, _t_x), (b, a, _t_y), (b, b, _t_hi))]
        + [(16, 16, _u)])


def _tp_a(s):
    return np.sqrt((s * (1 + s) * (3 + 2 * s)) / (1 + 2 * s)) / (1 + s)


def _tp_b(s):
    return ((-np.sqrt((1 + s) * (1 + 2 * s) * (3 + 2 * s)) + 2 * s * np.sqrt(2 + s + 1 / (1 + 2 * s)))
            / ((1 + s) * np.sqrt(3 + 2 * s)))


_T2P = ([(1, 1, _u)]
        + [r for a, b in ((2, 3), (4, 5)) for r in ((a, a, _tp_a), (b, a, _tp_b), (b, b, _u))]
        + [(6, 6, _u), (7, 7, _u), (8, 8, _u),
           (9, 9, lambda s: np.sqrt(-3 + 4 * s * (1 + s)) / (1 + 2 * s)),
           (10, 9, lambda s: -(np.sqrt(3 + 4 * s * (2 + s)) / ((1 + s) * (1 + 2 * s)))),
           (10, 10, lambda s: np.sqrt(s * (2 + s)) / (1 + s)),
           (11, 9, lambda s: 1 / (1 + 3 * s + 2 * s ** 2)),
           (11, 10, lambda s: -(1 / (1 + s))),
           (11, 11, _u)]
        + [r for a, b in ((12, 13), (14, 15)) for r in ((a, a, _tp_a), (b, a, _tp_b), (b, b, _u))]
        + [(16, 16, _u)])


def _tm_x(s):
    return 1 / np.sqrt(s * (1 + 2 * s))


def _tm_hi(s):
    return (1 / np.sqrt((s * (1 + s) * (1 + 2 * s)) / (-1 + 2 * s))
            + 1 / np.sqrt((s * (1 + s)) / (-1 + 4 * s ** 2))) / 2.


_T2M = ([(1, 1, _u)]
        + [r for a, b in ((2, 3), (4, 5)) for r in ((a, a, _u), (a, b, _tm_x), (b, b, _tm_hi))]
        + [(6, 6, _u), (7, 7, _u), (8, 8, _u),
           (9, 9, _u),
           (9, 10, lambda s: 1 / s),
           (9, 11, lambda s: 1 / (s + 2 * s ** 2)),
           (10, 10, lambda s: np.sqrt(-1 + s ** 2) / s),
           (10, 11, lambda s: np.sqrt(1 - 2 / (1 + 2 * s)) / s),
           (11, 11, lambda s: np.sqrt(-3 + 4 * s * (1 + s)) / (1 + 2 * s))]
        + [r for a, b in ((12, 13), (14, 15)) for r in ((a, a, _u), (a, b, _tm_x), (b, b, _tm_hi))]
        + [(16, 16, _u)])


# two-channel doublet rows (qs-2ch-doublet{p,m}.dat), functions of the spin of I1; combinations
# 2/4, 3/5, 12/14 and 13/15 carry the same factors
def _d_a(s):
    return (-2 * np.sqrt(s * (1 + s))) / (1 + 2 * s)


def _d_b(s):
    return 1 / (1 + 2 * s)


def _d_m1(s):
    return -1.0


_D2P = ([(1, 1, _u)]
        + [r for a, b in ((2, 3), (4, 5)) for r in ((a, a, _d_a), (b, a, _d_b), (b, b, _d_m1))]
        + [(6, 6, _u), (7, 7, _u), (8, 8, _u),
           (9, 9, lambda s: 1 / np.sqrt((s * (1 + 2 * s)) / (-1 + s + 2 * s ** 2))),
           (10, 9, lambda s: -(1 / np.sqrt(s * (1 + 2 * s)))),
           (10, 10, lambda s: (s * (3 + 2 * s)) / np.sqrt(s * (1 + s) * (3 + 4 * s * (2 + s)))),
           (11, 10, lambda s: -(1 / np.sqrt((1 + s) * (1 + 2 * s)))),
           (11, 11, _u)]
        + [r for a, b in ((12, 13), (14, 15)) for r in ((a, a, _d_a), (b, a, _d_b), (b, b, _d_m1))]
        + [(16, 16, _u)])


def _dm_c(s):
    return 1 / (-1 - 2 * s)


_D2M = ([(1, 1, _u)]
        + [r for a, b in ((2, 3), (4, 5)) for r in ((a, a, _d_m1), (a, b, _dm_c), (b, b, _d_a))]
        + [(6, 6, _u), (7, 7, _u), (8, 8, _u),
           (9, 9, _u),
           (9, 10, lambda s: 1 / np.sqrt(s * (1 + 2 * s))),
           (10, 10, lambda s: (-1 + s + 2 * s ** 2) / np.sqrt(s * (1 + s) * (-1 + 4 * s ** 2))),
           (10, 11, lambda s: 1 / np.sqrt((1 + s) * (1 + 2 * s))),
           (11, 11, lambda s: np.sqrt((s * (1 + 2 * s)) / ((1 + s) ** 3 * (3 + 2 * s)))
            + np.sqrt(s / ((1 + s) ** 3 * (3 + 4 * s * (2 + s)))) + np.sqrt(1 + 1 / (1 + s) - 6 / (3 + 2 * s)))]
        + [r for a, b in ((12, 13), (14, 15)) for r in ((a, a, _d_m1), (a, b, _dm_c), (b, b, _d_a))]
        + [(16, 16, _u)])


QS2 = Tables(
    2,
    IN=[(2, 0), (1, -1), (1, 1), (1, -1), (1, 1), (0, 0), (0, 0), (0, 0), (0, -2), (0, 0), (0, 2),
        (-1, -1), (-1, 1), (-1, -1), (-1, 1), (-2, 0)],
    QN=[(-2, 1), (-1, 2), (-1, 2), (-1, 2), (-1, 2), (0, 1), (0, 1), (0, 1), (0, 3), (0, 3), (0, 3),
        (1, 2), (1, 2), (1, 2), (1, 2), (2, 1)],
    OFFDIAG=[
        (1, 4, 0, _one),
        (1, 5, 0, _one),
        (2, 7, 0, lambda ss: -_a(ss)),
        (2, 9, 0, _one),
        (2, 10, 0, _b),
        (3, 7, 0, _b),
        (3, 10, 0, _a),
        (3, 11, 0, _one),
        (4, 8, 0, lambda ss: -(math.sqrt(2) * _a(ss))),
        (5, 8, 0, _b2),
        (6, 12, 0, _one),
        (6, 13, 0, _one),
        (7, 14, 0, lambda ss: -(1 / math.sqrt(2))),
        (7, 15, 0, lambda ss: -(1 / math.sqrt(2))),
        (9, 14, 0, lambda ss: -math.sqrt(1 - 1 / (2. * S(ss)))),
        (10, 14, 0, lambda ss: math.sqrt(1 + 1 / S(ss)) / math.sqrt(2)),
        (10, 15, 0, lambda ss: -(1 / math.sqrt(2 + 2 / S(ss)))),
        (11, 15, 0, lambda ss: math.sqrt(1 + 1 / (2 + 2 * S(ss)))),
        (12, 16, 0, lambda ss: -(math.sqrt(2) * _a(ss))),
        (13, 16, 0, _b2),
        (1, 2, 1, _one),
        (1, 3, 1, _one),
        (2, 6, 1, lambda ss: -(math.sqrt(2) * _a(ss))),
        (3, 6, 1, _b2),
        (4, 7, 1, lambda ss: -_a(ss)),
        (4, 9, 1, lambda ss: -1.0),
        (4, 10, 1, lambda ss: -_b(ss)),
        (5, 7, 1, _b),
        (5, 10, 1, lambda ss: -_a(ss)),
        (5, 11, 1, lambda ss: -1.0),
        (7, 12, 1, lambda ss: -(1 / math.sqrt(2))),
        (7, 13, 1, lambda ss: -(1 / math.sqrt(2))),
        (8, 14, 1, _one),
        (8, 15, 1, _one),
        (9, 12, 1, lambda ss: math.sqrt(1 - 1 / (2. * S(ss)))),
        (10, 12, 1, lambda ss: -(math.sqrt(1 + 1 / S(ss)) / math.sqrt(2))),
        (10, 13, 1, lambda ss: 1 / math.sqrt(2 + 2 / S(ss))),
        (11, 13, 1, lambda ss: -(math.sqrt(2 + 1 / (1 + S(ss))) / math.sqrt(2))),
        (14, 16, 1, lambda ss: -(math.sqrt(2) * _a(ss))),
        (15, 16, 1, _b2),
    ],
    DIAG=[(1, 0, 0.0), (2, 0, 0.0), (3, 0, 0.0), (4, 0, 1.0), (5, 0, 1.0), (6, 0, 0.0), (7, 0, 1.0), (8, 0, 2.0),
          (9, 0, 1.0), (10, 0, 1.0), (11, 0, 1.0), (12, 0, 1.0), (13, 0, 1.0), (14, 0, 2.0), (15, 0, 2.0),
          (16, 0, 2.0),
          (1, 1, 0.0), (2, 1, 1.0), (3, 1, 1.0), (4, 1, 0.0), (5, 1, 0.0), (6, 1, 2.0), (7, 1, 1.0), (8, 1, 0.0),
          (9, 1, 1.0), (10, 1, 1.0), (11, 1, 1.0), (12, 1, 2.0), (13, 1, 2.0), (14, 1, 1.0), (15, 1, 1.0),
          (16, 1, 2.0)],
    DIAG_FIRST=True,
    RECALC_F=[
        ((1, 1), 0, [(4, 1, _one),
                     (7, 3, lambda s: -math.sqrt(2 - 1 / (1 + S(s))) / 2.),
                     (8, 5, lambda s: -_c(s)),
                     (9, 2, lambda s: -1.0),
                     (10, 3, lambda s: -math.sqrt(2 + 1 / (1 + S(s))) / 2.),
                     (12, 6, _one),
                     (14, 7, lambda s: -(1 / math.sqrt(2))),
                     (14, 10, lambda s: S(s) / (math.sqrt(2) * math.sqrt(S(s) * (1 + S(s))))),
                     (15, 11, _c),
                     (16, 13, lambda s: -_c(s))]),
        ((1, 1), 1, [(2, 1, _one),
                     (6, 3, lambda s: -_c(s)),
                     (7, 5, lambda s: -math.sqrt(2 - 1 / (1 + S(s))) / 2.),
                     (9, 4, _one),
                     (10, 5, lambda s: math.sqrt(2 + 1 / (1 + S(s))) / 2.),
                     (12, 7, lambda s: -(1 / math.sqrt(2))),
                     (12, 10, lambda s: -(S(s) / (math.sqrt(2) * math.sqrt(S(s) * (1 + S(s)))))),
                     (13, 11, lambda s: -_c(s)),
                     (14, 8, _one),
                     (16, 15, lambda s: -_c(s))]),
        ((1, -1), 0, [(5, 1, _one),
                      (7, 2, lambda s: math.sqrt(2 + 1 / S(s)) / 2.),
                      (8, 4, lambda s: math.sqrt(1 + 1 / (2. * S(s)))),
                      (10, 2, lambda s: -math.sqrt(2 - 1 / S(s)) / 2.),
                      (11, 3, lambda s: -1.0),
                      (13, 6, _one),
                      (14, 9, lambda s: -(math.sqrt(2 + 1 / S(s)) / math.sqrt(2))),
                      (15, 7, lambda s: -(1 / math.sqrt(2))),
                      (15, 10, lambda s: -(math.sqrt(1 + 1 / S(s)) / math.sqrt(2))),
                      (16, 12, lambda s: math.sqrt(1 + 1 / (2. * S(s))))]),
        ((1, -1), 1, [(3, 1, _one),
                      (6, 2, lambda s: math.sqrt(1 + 1 / (2. * S(s)))),
                      (7, 4, lambda s: math.sqrt(2 + 1 / S(s)) / 2.),
                      (10, 4, lambda s: math.sqrt(2 - 1 / S(s)) / 2.),
                      (11, 5, _one),
                      (12, 9, lambda s: math.sqrt(1 + 1 / (2. * S(s)))),
                      (13, 7, lambda s: -(1 / math.sqrt(2))),
                      (13, 10, lambda s: math.sqrt(1 + 1 / S(s)) / math.sqrt(2)),
                      (15, 8, _one),
                      (16, 14, lambda s: math.sqrt(1 + 1 / (2. * S(s))))]),
    ],
    DOUBLET=[((-1, 1), _D2P), ((-1, -1), _D2M)],
    TRIPLET=[
        ((0, 0), _T2S),
        ((0, 2), _T2P),
        ((0, -2), _T2M),
    ],
    doublet_of_spin=True,
)


def tables(channels: int) -> Tables:
    if channels == 1:
        return QS1
    if channels == 2:
        return QS2
    raise ValueError(f"QS with {channels} channels is not supported")
