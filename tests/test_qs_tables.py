"""The QS coefficient tables of nrgljubljana_b200/qs.py against the reference's own tables
(c++/symmetry/coefnew/qs/qs-{1,2}ch-*.dat), evaluated for SS = 1..11 by
tests/golden/make_qs_tables.py into tests/golden/qs_tables.json: every row in the
reference's order, every factor to 1e-14 relative wherever the reference's value is finite,
and non-finite (or an error) wherever it is not -- a row is only ever used where its value is
finite."""
import json
import math
import os

import numpy as np
import pytest

from nrgljubljana_b200 import qs

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "qs_tables.json")) as f:
    REF = json.load(f)
SS = REF["ss"]


def ours(fn, ss):
    """A factor evaluated the way the run evaluates it (qs.ieee); non-finite values, and the
    error triplet_factor raises for them, as nan."""
    try:
        v = qs.ieee(fn, ss)
    except AssertionError:
        return math.nan
    return v if math.isfinite(v) else math.nan


def check_values(got, want, what):
    for ss, g, w in zip(SS, got, want):
        if math.isfinite(w):
            assert math.isfinite(g) and abs(g - w) <= 1e-14 * max(1.0, abs(w)), (what, ss, g, w)
        else:
            assert not math.isfinite(g), (what, ss, g, w)


TABLES = [(1, qs.QS1), (2, qs.QS2)]


@pytest.mark.parametrize("ch,T", TABLES)
def test_offdiag_and_diag(ch, T):
    ref = REF[f"{ch}ch-offdiag"]
    assert [(i, j, c) for i, j, c, _ in ref] == [(i, j, c) for i, j, c, _ in T.OFFDIAG]
    for (i, j, c, vals), (_, _, _, fn) in zip(ref, T.OFFDIAG):
        check_values([ours(fn, ss) for ss in SS], vals, f"offdiag {i},{j},{c}")
    assert [tuple(r) for r in REF[f"{ch}ch-diag"]] == [(i, c, float(nu)) for i, c, nu in T.DIAG]


@pytest.mark.parametrize("ch,T", TABLES)
def test_recalc_f(ch, T):
    files = {((1, 1), 0): "spinupa", ((1, -1), 0): "spindowna", ((1, 1), 1): "spinupb", ((1, -1), 1): "spindownb"}
    assert len(T.RECALC_F) == 2 * ch
    for dq, c, rows in T.RECALC_F:
        ref = REF[f"{ch}ch-{files[(dq, c)]}"]
        assert [(a, b) for a, b, _ in ref] == [(a, b) for a, b, _ in rows]
        for (a, b, vals), (_, _, fn) in zip(ref, rows):
            check_values([ours(fn, ss) for ss in SS], vals, f"recalc_f {dq} ch{c} {a},{b}")


@pytest.mark.parametrize("ch,T", TABLES)
def test_doublet_and_triplet(ch, T):
    for tables, names, factor in ((T.DOUBLET, ("doubletp", "doubletm"), T.doublet_factor),
                                  (T.TRIPLET, ("triplets", "tripletp", "tripletm"), qs.triplet_factor)):
        assert len(tables) == len(names)
        for (dq, rows), name in zip(tables, names):
            ref = REF[f"{ch}ch-{name}"]
            assert [(a, b) for a, b, _ in ref] == [(a, b) for a, b, _ in rows], name
            for (a, b, vals), (_, _, fn) in zip(ref, rows):
                check_values([ours(lambda s, fn=fn: factor(fn, s), ss) for ss in SS], vals, f"{name} {a},{b}")


def test_table_shapes():
    for ch, T in TABLES:
        assert T.COMBS == len(T.IN) == len(T.QN) == 4 ** ch
    assert np.array_equal(np.array(qs.QS1.IN), np.array([(1, 0), (0, -1), (0, 1), (-1, 0)]))


def test_global_charge_tables():
    """Q1, Q2, Qdiff, Qtot of two-channel QS row by row (qs-2ch-{q1,q2,qdiff,qtot}.dat);
    one channel has no global operators (recalc_global asserts, nrg-recalc-QS.hpp:680-740)."""
    assert sorted(qs.QS2.GLOBAL) == ["Q1", "Q2", "Qdiff", "Qtot"]
    for name, rows in qs.QS2.GLOBAL.items():
        assert [tuple(r) for r in REF[f"2ch-{name.lower()}"]] == rows, name
    assert qs.QS1.GLOBAL == {}
