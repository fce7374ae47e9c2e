"""Pins the CPU oracle to the known-answer tests of the reference's own unit tests.

Every expected value below is read from the reference test sources (cited per test);
the oracle must reproduce them exactly as the reference's gtest EXPECT_DOUBLE_EQ does
(4 ulp), or to the tolerance stated.
"""
import math

import numpy as np
import pytest

SQ2 = 1.0 / math.sqrt(2.0)


def ulp_eq(a, b, ulps=4):
    return a == b or abs(a - b) <= ulps * np.spacing(max(abs(a), abs(b)))


@pytest.mark.parametrize("solver", ["dsyev", "dsyevd", "dsyevr"])
def test_pauli_z(oracle, solver):
    # test/unit/diag_test/diag_test.cpp:83-97 (dsyev), 119-131 (dsyevr), 155-167 (dsyevd)
    m = np.array([[-1.0, 0.0], [0.0, 1.0]])
    val, vec = oracle.diagonalise(m, solver)
    assert len(val) == 2 and vec.shape == (2, 2)
    assert ulp_eq(val[0], -1.0) and ulp_eq(val[1], 1.0)
    assert ulp_eq(abs(vec[0, 0]), 1.0) and vec[0, 1] == 0.0
    assert vec[1, 0] == 0.0 and ulp_eq(abs(vec[1, 1]), 1.0)


@pytest.mark.parametrize("solver", ["dsyev", "dsyevd", "dsyevr"])
def test_pauli_x_upper_only(oracle, solver):
    # test/unit/diag_test/diag_test.cpp:98-112: only m(0,1) set; the upper triangle is read
    m = np.array([[0.0, 1.0], [0.0, 0.0]])
    val, vec = oracle.diagonalise(m, solver)
    assert ulp_eq(val[0], -1.0) and ulp_eq(val[1], 1.0)
    assert ulp_eq(abs(vec[0, 0]), SQ2) and ulp_eq(abs(vec[0, 1]), SQ2)
    assert ulp_eq(vec[0, 0] * vec[0, 1], -0.5)
    assert ulp_eq(abs(vec[1, 0]), SQ2) and ulp_eq(abs(vec[1, 1]), SQ2)
    assert ulp_eq(vec[1, 0] * vec[1, 1], 0.5)


def test_copy_results_identity_is_unitary(oracle):
    # test/unit/diag_test/diag_test.cpp:60-66
    assert oracle.is_unitary(np.eye(2))


def test_is_unitary_cases(oracle):
    # test/unit/numerics/numerics.cpp:147-171
    assert oracle.is_unitary(np.eye(2))
    assert not oracle.is_unitary(np.zeros((2, 2)))
    assert not oracle.is_unitary(np.array([[1.0, SQ2], [0.0, SQ2]]))
    assert not oracle.is_unitary(np.array([[1.0, 0.0], [SQ2, SQ2]]))


def test_product_transform_rotate_all_ones(oracle):
    # test/unit/numerics/numerics.cpp:491-545 (expected 2, 4, 4, 2, 2)
    one = np.ones((2, 2))
    r = np.zeros((2, 2)); oracle.product(r, 1.0, one, one); assert (r == 2).all()
    r = np.zeros((2, 2)); oracle.transform(r, 1.0, one, one, one); assert (r == 4).all()
    r = np.zeros((2, 2)); oracle.rotate(r, 1.0, one, one); assert (r == 4).all()
    assert (oracle.matmul(one, one) == 2).all()
    assert (oracle.matmul(one.T.copy(), one) == 2).all()  # matrix_adj_prod, real case


def test_prod_fit(oracle):
    # test/unit/numerics/numerics.cpp:321-404
    a = np.full((2, 2), 2.0); b = np.full((1, 1), 2.0)
    m = oracle.prod_fit(a, b); assert m.shape == (2, 1) and (m == 4).all()       # prod_fit_left
    a1 = np.full((1, 1), 2.0); b2 = np.full((2, 2), 2.0)
    m = oracle.prod_fit(a1, b2); assert m.shape == (1, 2) and (m == 4).all()     # prod_fit_right
    a = np.array([[1.0, 2.0], [3.0, 4.0]])
    assert (oracle.prod_fit(a, a) == np.array([[7.0, 10.0], [15.0, 22.0]])).all()


def test_chit_weight(oracle):
    # test/unit/numerics/numerics.cpp:443-449
    assert ulp_eq(oracle.chit_weight(2.0, 1.0, 1.0), math.exp(-1.0) - math.exp(-2.0))
    assert ulp_eq(oracle.chit_weight(2.0, 1.0, 0.5), (math.exp(-0.5) - math.exp(-1.0)) / 0.5)
    assert ulp_eq(oracle.chit_weight(1.0, 1.0, 1.0), math.exp(-1.0))
    assert ulp_eq(oracle.chit_weight(3.0, 1.0, 1.0), (math.exp(-1.0) - math.exp(-3.0)) / 2.0)
    assert ulp_eq(oracle.chit_weight(3.0, 3.0, 1.0), math.exp(-3.0))


def test_transform_complexity_matches_numpy(oracle):
    # Cross-check of the strided GEMM leaves against numpy on random data.
    rng = np.random.default_rng(7)
    A, O, B = rng.standard_normal((5, 3)), rng.standard_normal((3, 4)), rng.standard_normal((6, 4))
    M = rng.standard_normal((5, 6)); ref = M + 0.7 * A @ O @ B.T
    oracle.transform(M, 0.7, A, O, B)
    assert np.allclose(M, ref, rtol=1e-13, atol=1e-13)
    U, R = rng.standard_normal((4, 7)), rng.standard_normal((4, 4))
    M = np.zeros((7, 7)); oracle.rotate(M, 1.5, U, R)
    assert np.allclose(M, 1.5 * U.T @ R @ U, rtol=1e-13, atol=1e-13)


def test_loggrid_and_add_std(oracle):
    # bins.hpp:95-132: 10 bins per decade from 1e-10 to 1 gives 101 points; a peak at a grid
    # point lands in one bin; one between points is split linearly in log10 E.
    cb = oracle.ChainBinning(-10.0, 0.0, 10)
    assert cb.nbins == 101
    assert ulp_eq(cb.energies[0], 1e-10) and ulp_eq(cb.energies[-1], 1.0)
    cb.add(np.array([1e-5]), np.array([2.0]))
    i = int(np.argmax(cb.pos_re))
    assert i == 50 and abs(cb.pos_re.sum() - 2.0) < 1e-15
    cb2 = oracle.ChainBinning(-10.0, 0.0, 10)
    e = 10 ** (-5 + 0.25 / 10)
    cb2.add(np.array([-e, 1e-20, 5.0, 1e-12]), np.array([1.0, 3.0, 4.0, 5.0]))
    assert abs(cb2.neg_re[50] - 0.75) < 1e-12 and abs(cb2.neg_re[51] - 0.25) < 1e-12
    assert cb2.pos_re[0] == 3.0 + 5.0      # below zero_epsilon and below emin -> first bin
    assert cb2.pos_re[-1] == 4.0           # above emax -> last bin


def test_windowfunction(oracle):
    # spectrum.hpp:91-109: linear window f(0)=0, f(1)=1; exceptions for first/last steps.
    assert oracle.windowfunction(1.5, 1.0, 2.0, 4.0) == 0.5
    assert oracle.windowfunction(3.0, 1.0, 2.0, 4.0) == 0.5
    assert oracle.windowfunction(0.5, 1.0, 2.0, 4.0) == 0.0
    assert oracle.windowfunction(0.5, 1.0, 2.0, 4.0, last=True) == 1.0
    assert oracle.windowfunction(5.0, 1.0, 2.0, 4.0, first=True) == 1.0


def test_batch_matches_single(oracle):
    rng = np.random.default_rng(3)
    blocks = []
    for n in (1, 2, 5, 17, 40):
        h = rng.standard_normal((n, n)); h = np.triu(h + h.T)
        blocks.append(h)
    ev, vec = oracle.diag_batch(blocks, nthreads=2)
    for h, w, v in zip(blocks, ev, vec):
        w1, v1 = oracle.diagonalise(h)
        assert np.array_equal(w, w1)
        assert oracle.is_unitary(v)
        full = np.triu(h) + np.triu(h, 1).T
        assert np.allclose(v @ full @ v.T, np.diag(w), atol=1e-12 * max(1.0, np.abs(w).max()))
