"""The oracle's vectorised Matsubara terms (oracle/nrg_run_cpu.py: mats_pair, dmnrg_mats_pair,
ft_mats_pair) against a term-by-term loop in the reference's order and form
(c++/algo_FDM.hpp:167-217, c++/algo_DMNRG.hpp:76-100, c++/algo_FT.hpp:63-85), on random pairs
with exact degeneracies, so that the bosonic n = 0 limits (|E| <= 1e-8) are exercised, for both
statistics."""
import math

import numpy as np
import pytest

WEIGHT_TOL = 1e-8


def ww(n, sign, T):
    return T * math.pi * (2 * n + (0 if sign == 1 else 1))


def loop_fdm(EGi, Ki, EGj, Kj, o1, o2, rho_i, rho_j, factor, sign, T, wnf, mats):
    ni, nj = len(EGi), len(EGj)
    rho_op2 = rho_j @ o2[:rho_j.shape[0], :]
    op2_rho = o2[:, :rho_i.shape[0]] @ rho_i
    G = np.zeros(mats, dtype=complex)
    for i in range(Ki, ni):
        for j in range(Kj, nj):
            E = EGj[j] - EGi[i]
            wA = o1[j, i] * o2[j, i] * wnf * math.exp(-EGi[i] / T)
            wB = o1[j, i] * o2[j, i] * (-sign) * wnf * math.exp(-EGj[j] / T)
            for n in range(mats):
                if sign == -1 or n > 0 or abs(E) > WEIGHT_TOL:
                    G[n] += factor * (wA + wB) / (ww(n, sign, T) * 1j - E)
                else:
                    G[n] += factor * (-wA / T)
    for i in range(Ki, ni):
        for j in range(Kj):
            E = EGj[j] - EGi[i]
            wA = o1[j, i] * o2[j, i] * wnf * math.exp(-EGi[i] / T)
            wB = o1[j, i] * rho_op2[j, i] * (-sign)
            for n in range(mats):
                G[n] += factor * (wA + wB) / (ww(n, sign, T) * 1j - E)
    for i in range(Ki):
        for j in range(Kj, nj):
            E = EGj[j] - EGi[i]
            wA = o1[j, i] * op2_rho[j, i]
            wB = (-sign) * o1[j, i] * o2[j, i] * wnf * math.exp(-EGj[j] / T)
            for n in range(mats):
                G[n] += factor * (wA + wB) / (ww(n, sign, T) * 1j - E)
    return G


def loop_dmnrg(Em, Ej, o1, o2, rho_p, rho_1, factor, sign, T, mats):
    G = np.zeros(mats, dtype=complex)
    for rm in range(len(Em)):
        for rj in range(len(Ej)):
            wA = sum(o2[rj, ri] * rho_p[rm, ri] for ri in range(len(Em))) * o1[rj, rm]
            wB = sum(o1[ri, rm] * rho_1[rj, ri] for ri in range(len(Ej))) * o2[rj, rm]
            E = Ej[rj] - Em[rm]
            for n in range(mats):
                if sign == -1 or n > 0 or abs(E) > WEIGHT_TOL:
                    G[n] += factor * (wA + (-sign) * wB) / (ww(n, sign, T) * 1j - E)
                else:
                    G[n] += factor * (-wA / T)
    return G


def loop_ft(Ep, E1, o1, o2, Z, factor, sign, T, mats):
    G = np.zeros(mats, dtype=complex)
    beta = 1.0 / T
    for r1 in range(len(E1)):
        for rp in range(len(Ep)):
            E = E1[r1] - Ep[rp]
            for n in range(mats):
                if sign == -1 or n > 0 or abs(E) > WEIGHT_TOL:
                    sf = ((-sign) * math.exp(-beta * E1[r1]) + math.exp(-beta * Ep[rp])) / (Z * (ww(n, sign, T) * 1j - E))
                else:
                    sf = -math.exp(-beta * E1[r1]) / (Z * T)
                G[n] += factor * o1[r1, rp] * o2[r1, rp] * sf
    return G


def degenerate_levels(rng, n):
    e = np.sort(rng.uniform(0.0, 2.0, n))
    e[1::3] = e[0::3][:len(e[1::3])]  # exact repeats
    return np.sort(e)


@pytest.mark.parametrize("sign", [1, -1])
def test_fdm_mats_terms(sign):
    from oracle.nrg_run_cpu import mats_pair
    rng = np.random.default_rng(11 + sign)
    ni, nj, Ki, Kj, mats, T = 7, 6, 3, 2, 5, 0.3
    EGi, EGj = np.sort(rng.uniform(0.0, 2.0, ni)), np.sort(rng.uniform(0.0, 2.0, nj))
    # equal energies across the pair in the D x D sector only: the reference divides by
    # i w_0 - E = 0 in the D x K and K x D terms of a bosonic operator (no limit there)
    EGj[Kj:Kj + 2] = EGi[Ki:Ki + 2]
    o1, o2 = rng.standard_normal((nj, ni)), rng.standard_normal((nj, ni))
    rho_i, rho_j = rng.standard_normal((Ki, Ki)), rng.standard_normal((Kj, Kj))
    w = np.array([ww(n, sign, T) for n in range(mats)])
    got = mats_pair(EGi, Ki, EGj, Kj, o1, o2, rho_i, rho_j, 0.7, sign, T, 0.4, w)
    want = loop_fdm(EGi, Ki, EGj, Kj, o1, o2, rho_i, rho_j, 0.7, sign, T, 0.4, mats)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("sign", [1, -1])
def test_dmnrg_mats_terms(sign):
    from oracle.nrg_run_cpu import dmnrg_mats_pair
    rng = np.random.default_rng(21 + sign)
    ki, kj, mats, T = 5, 4, 4, 0.2
    Em, Ej = degenerate_levels(rng, ki), degenerate_levels(rng, kj)
    Ej[:2] = Em[:2]
    o1, o2 = rng.standard_normal((kj, ki)), rng.standard_normal((kj, ki))
    rp = rng.standard_normal((ki, ki))
    r1 = rng.standard_normal((kj, kj))
    w = np.array([ww(n, sign, T) for n in range(mats)])
    got = dmnrg_mats_pair(Em, Ej, o1, o2, rp + rp.T, r1 + r1.T, 1.3, sign, T, w)
    want = loop_dmnrg(Em, Ej, o1, o2, rp + rp.T, r1 + r1.T, 1.3, sign, T, mats)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("sign", [1, -1])
def test_ft_mats_terms(sign):
    from oracle.nrg_run_cpu import ft_mats_pair
    rng = np.random.default_rng(31 + sign)
    kp, k1, mats, T = 6, 5, 4, 0.25
    Ep, E1 = degenerate_levels(rng, kp), degenerate_levels(rng, k1)
    E1[:2] = Ep[:2]
    o1, o2 = rng.standard_normal((k1, kp)), rng.standard_normal((k1, kp))
    w = np.array([ww(n, sign, T) for n in range(mats)])
    got = ft_mats_pair(Ep, E1, o1, o2, 2.5, 0.9, sign, T, w)
    want = loop_ft(Ep, E1, o1, o2, 2.5, 0.9, sign, T, mats)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
