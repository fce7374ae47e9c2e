"""The extended-precision sums of the FDM thermodynamics (nrgljubljana_b200/ddsum.py) against
exact rational arithmetic, including the cancellation that <E^2> - <E>^2 suffers at low
temperature."""
import math
from fractions import Fraction

import numpy as np

from nrgljubljana_b200 import ddsum


def exact_dot(d, e, power=1):
    return sum((Fraction(float(x)) * Fraction(float(y)) ** power for x, y in zip(d, e)), Fraction(0))


def test_two_prod_is_exact():
    rng = np.random.default_rng(1)
    a = rng.standard_normal(1000) * 10.0 ** rng.integers(-30, 30, 1000)
    b = rng.standard_normal(1000) * 10.0 ** rng.integers(-30, 30, 1000)
    p, e = ddsum.two_prod(a, b)
    for x, y, pp, ee in zip(a, b, p, e):
        assert Fraction(float(pp)) + Fraction(float(ee)) == Fraction(float(x)) * Fraction(float(y))


def test_sums_match_exact_arithmetic():
    rng = np.random.default_rng(2)
    d = np.exp(-rng.uniform(0, 40, 5000))          # Boltzmann-like weights over many decades
    e = -3.6 + rng.uniform(0, 1e-5, 5000)           # energies close to a large offset
    for got, want in ((ddsum.dot(d, e), exact_dot(d, e)), (ddsum.dot_sq(d, e), exact_dot(d, e, 2)),
                      (ddsum.exact_sum([d, e]), sum((Fraction(float(x)) for x in np.concatenate([d, e])),
                                                    Fraction(0)))):
        assert abs(got - want) <= abs(want) * Fraction(1, 2 ** 100)


def test_variance_survives_cancellation():
    """Var = <e^2> - <e>^2 with <e> ~ 3.6 and Var ~ 1e-16: a double sum loses it entirely,
    the double-double one keeps it to a few parts in 1e6."""
    rng = np.random.default_rng(3)
    w = rng.uniform(0.5, 1.0, 2000)
    w = w / math.fsum(w)
    e = -3.6 + rng.standard_normal(2000) * 1e-8
    m1, m2 = ddsum.dot(w, e), ddsum.dot_sq(w, e)
    var = float(m2 - m1 * m1)
    ex1, ex2 = exact_dot(w, e), exact_dot(w, e, 2)
    exact = float(ex2 - ex1 * ex1)
    assert exact > 0 and abs(var - exact) <= 1e-6 * exact
    naive = float(np.sum(w * e * e) - np.sum(w * e) ** 2)
    assert abs(naive - exact) > 1e-3 * exact  # the plain double sum is off
