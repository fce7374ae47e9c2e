"""Extended-precision sums for the FDM thermodynamics of a run.

The reference accumulates the partial statistical sums and the energy moments of the FDM
thermodynamics in 400-bit GMP (calc_ZnD and fdm_thermodynamics, c++/measurements.hpp:60-163),
because the heat capacity C = (<E^2> - <E>^2) / T^2 cancels almost all digits of its two
terms at low temperature. The terms themselves are doubles. Here every product of doubles is
split exactly into two doubles (Dekker's product), every sum of doubles is taken exactly and
rounded once to a double-double with math.fsum, and the few per-step quotients are combined
as exact rationals: the result agrees with the 400-bit computation to about 2^-106 relative
in <E> and <E^2>. Host-side, O(states) numpy work.
"""
from __future__ import annotations

import math
from fractions import Fraction
from typing import Iterable, Tuple

import numpy as np

_SPLIT = 134217729.0  # 2^27 + 1


def two_prod(a: np.ndarray, b: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """p, e with p + e = a * b exactly (Dekker's product without FMA; |a|, |b| < 2^996)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    p = a * b
    t = _SPLIT * a
    ah = t - (t - a)
    al = a - ah
    t = _SPLIT * b
    bh = t - (t - b)
    bl = b - bh
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def exact_sum(parts: Iterable[np.ndarray]) -> Fraction:
    """The sum of all elements of `parts`, rounded to a double-double and returned exactly."""
    vals = np.concatenate([np.ravel(np.asarray(x, dtype=np.float64)) for x in parts] or [np.zeros(0)])
    hi = math.fsum(vals)
    lo = math.fsum(np.append(vals, -hi))
    return Fraction(hi) + Fraction(lo)


def dot(d: np.ndarray, e: np.ndarray) -> Fraction:
    """sum_i d_i e_i to double-double accuracy."""
    p, err = two_prod(d, e)
    return exact_sum((p, err))


def dot_sq(d: np.ndarray, e: np.ndarray) -> Fraction:
    """sum_i d_i e_i^2 to double-double accuracy."""
    q, qe = two_prod(e, e)
    p, pe = two_prod(d, q)
    return exact_sum((p, pe, np.asarray(d, dtype=np.float64) * qe))
