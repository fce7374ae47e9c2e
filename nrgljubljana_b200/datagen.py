"""Generator of NRG Ljubljana ``data`` files (the initial cluster and the Wilson chain).

Restates, for the single-impurity Anderson model with symmetry QS and a flat band, what
the reference's Mathematica front end (nrginit) writes:

* Wilson-chain coefficients xi_n, zeta_n: the discretisation of the flat band (schemes Z,
  C and Y with twist z; nrginit/initial.m:2767-2781, 3418-3524) and the Lanczos recursion
  of Chen and Jayaprakash (nrginit/initial.m:2925-3040, "tri=old"), run in fixed point on
  Python integers with about the reference's 1000 digits of precision.
* The initial cluster: impurity d and the first chain site f0, H = delta n_d +
  U/2 (n_d - 1)^2 + V sum_sigma (f0^dag d + d^dag f0) + zeta_0 (n_f0 - 1) with
  V = sqrt(theta0 A_Lambda / pi), theta0 = 2 Gamma (nrginit/initial.m:448-470, 505-509,
  543-640, 816-827; A_Lambda = 1 for Z and C, (1+1/L)/(1-1/L) ln(L)/2 for Y,
  nrginit/initial.m:996).
* Its QS multiplets (charge Q = N - 2, spin S, SS = 2S+1), energies minus the ground-state
  energy divided by SCALE(0) (nrginit/initial.m:983, 3986-3992), the reduced matrix elements
  of f0^dag and of the requested operators. Reduced matrix elements follow the
  Wigner-Eckart convention <j' m'| T_q |j m> = <j m; k q | j' m'> <j'||T||j> with
  Condon-Shortley Clebsch-Gordan coefficients -- the convention the QS recalculation
  tables (qs-1ch-spinupa/spindowna.dat) assume.

The text produced is read back by ``inputs.read_data``; host-side, no device work.
"""
from __future__ import annotations

import math
from math import isqrt
from typing import Dict, List, Sequence, Tuple

import numpy as np

Invar = Tuple[int, int]


# ------------------------------------------------------------------ Wilson chain
def wilson_chain(Lambda: float, nmax: int, z: float = 1.0, discretization: str = "Z", mmax: int = -1,
                 bits: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """xi_n, zeta_n for n = 0..nmax of a flat band of half-width 1.

    The discretisation constants are evaluated with mpmath; the Lanczos recursion runs in
    fixed point on Python integers with `bits` fraction bits. The recursion loses about ten
    decimal digits per site (a 100-site chain needs the reference's 1000 digits), so the
    default is 34 bits per site plus 800. Every fixed-point product and quotient is
    truncated toward zero, an odd function, so the recursion stays exactly odd in the band
    energy and a particle-hole symmetric band gives zeta = 0 exactly. Results are rounded
    once to double."""
    import mpmath as mp
    if mmax < 0:
        mmax = max(80, 2 * nmax)  # nrginit/initial.m:2745
    if bits <= 0:
        bits = 34 * nmax + 800
    old = mp.mp.dps
    mp.mp.dps = int(bits * 0.30103) + 20
    try:
        L = mp.mpf(Lambda)
        Z = mp.mpf(z)
        lnL = mp.log(L)
        eps = [mp.mpf(1)] + [L ** (-Z - m + 1) for m in range(1, mmax + 2)]
        df = [eps[m] - eps[m + 1] for m in range(mmax + 1)]
        if discretization == "Z":
            de = [(1 - L ** (-Z) + lnL - Z * lnL) / lnL] + \
                 [(eps[m] - eps[m + 1]) / mp.log(eps[m] / eps[m + 1]) for m in range(1, mmax + 1)]
        elif discretization == "C":
            de = [(eps[m] - eps[m + 1]) / mp.log(eps[m] / eps[m + 1]) for m in range(mmax + 1)]
        elif discretization == "Y":
            de = [(1 + L ** (-Z)) / 2] + [(1 + 1 / L) / 2 * L ** (1 - Z - m) for m in range(1, mmax + 1)]
        else:
            raise ValueError(f"discretization {discretization!r}")
        theta = mp.mpf(2)
        u0 = [mp.sqrt(x / theta) for x in df]
        norm = mp.sqrt(mp.fsum(2 * x * x for x in u0))  # du and dv start equal (p-h symmetric band)
        scale = mp.mpf(2) ** bits
        de_i = np.array([int(mp.nint(x * scale)) for x in de], dtype=object)
        up = np.array([int(mp.nint(x / norm * scale)) for x in u0], dtype=object)
    finally:
        mp.mp.dps = old
    B = bits
    ONE = 1 << B

    def shr(a):  # a / 2^B truncated toward zero
        if isinstance(a, np.ndarray):
            return np.where(a < 0, -((-a) >> B), a >> B)
        return -((-a) >> B) if a < 0 else a >> B

    def div(a, x):  # a / x in fixed point (x > 0), truncated toward zero
        return np.where(a < 0, -((-a) * ONE // x), a * ONE // x)

    de2 = shr(de_i * de_i)
    vp = up.copy()
    zero = np.array([0] * (mmax + 1), dtype=object)
    up_prev, vp_prev = zero.copy(), zero.copy()
    xi_prev = xi2_prev = 0
    xis, zetas = [], []
    for n in range(nmax + 1):
        u2, v2 = shr(up * up), shr(vp * vp)
        zeta = int(shr(de_i * u2).sum()) - int(shr(de_i * v2).sum())
        xi2 = int(shr(de2 * (u2 + v2)).sum()) - xi2_prev - shr(zeta * zeta)
        if xi2 <= 0:
            raise ArithmeticError(f"Lanczos recursion lost precision at site {n}; raise bits")
        xi = isqrt(xi2 << B)
        xis.append(xi / ONE)
        zetas.append(zeta / ONE)
        nu = div(shr((de_i - zeta) * up) - shr(xi_prev * up_prev), xi)
        nv = div(shr((-de_i - zeta) * vp) - shr(xi_prev * vp_prev), xi)
        up_prev, vp_prev, up, vp = up, vp, nu, nv
        xi_prev, xi2_prev = xi, xi2
    return np.array(xis), np.array(zetas)


def scale0(Lambda: float, z: float = 1.0, discretization: str = "Z", bandrescale: float = 1.0) -> float:
    """SCALE[0] of nrginit/initial.m:976-983 (equal to the run driver's SCALE(0))."""
    if discretization == "Y":
        sc0 = (1 + 1 / Lambda) / 2 * Lambda ** -(z - 1)
    else:
        sc0 = (1 - 1 / Lambda) / math.log(Lambda) * Lambda ** -(z - 1)
    return sc0 * Lambda ** (1 / 2) * bandrescale


def gamma_A(Lambda: float, discretization: str) -> float:
    """Lambda correction of the hybridisation for scheme Y (nrginit/initial.m:996)."""
    return 0.5 * (1 + 1 / Lambda) / (1 - 1 / Lambda) * math.log(Lambda) if discretization == "Y" else 1.0


# ------------------------------------------------------------------ Fock space of d and f0
# modes 0: d up, 1: d down, 2: f0 up, 3: f0 down; Jordan-Wigner ordering
_NM = 4


def _annihilators() -> List[np.ndarray]:
    dim = 1 << _NM
    ops = []
    for k in range(_NM):
        c = np.zeros((dim, dim))
        for s in range(dim):
            if s >> k & 1:
                sign = -1.0 if bin(s & ((1 << k) - 1)).count("1") % 2 else 1.0
                c[s ^ (1 << k), s] = sign
        ops.append(c)
    return ops


def _highest_weight(states: np.ndarray, Splus: np.ndarray) -> np.ndarray:
    """Orthonormal basis of the kernel of S+ inside span(states) (columns)."""
    M = Splus @ states
    _, s, vt = np.linalg.svd(M, full_matrices=True)
    rank = int(np.sum(s > 1e-10))
    return states @ vt[rank:].T


def siam_qs(U: float, delta: float, Gamma: float, Lambda: float, nmax: int, z: float = 1.0,
            discretization: str = "Z", ops: Sequence[str] = ("n_d",), xi=None, zeta=None) -> str:
    """The ``data`` file of the QS single-impurity Anderson model (one channel, flat band).

    delta = eps_d + U/2. Operators: singlets n_d, n_d^2, I, Himp, Hhyb, hop0 and the doublet
    A_d (d^dag)."""
    if xi is None or zeta is None:
        xi, zeta = wilson_chain(Lambda, nmax, z, discretization)
    c = _annihilators()
    cd = [m.T for m in c]
    n = [cd[k] @ c[k] for k in range(_NM)]
    nd = n[0] + n[1]
    nf = n[2] + n[3]
    I = np.eye(1 << _NM)
    V = math.sqrt(2.0 * Gamma * gamma_A(Lambda, discretization) / math.pi)
    hop0 = sum(cd[2 + s] @ c[s] + cd[s] @ c[2 + s] for s in (0, 1))
    Himp = delta * nd + U / 2 * (nd - I) @ (nd - I)
    H = Himp + V * hop0 + zeta[0] * (nf - I)
    Sp = cd[0] @ c[1] + cd[2] @ c[3]   # S+ = sum over sites of c_up^dag c_down
    Sm = Sp.T
    diagN = np.round(np.diag(nd + nf)).astype(int)
    diag2Sz = np.round(np.diag(n[0] - n[1] + n[2] - n[3])).astype(int)
    sc = scale0(Lambda, z, discretization)
    # multiplets: the highest-weight states of each (N, S), diagonalised
    subs: Dict[Invar, Tuple[np.ndarray, np.ndarray]] = {}
    for N in range(0, 5):
        for twoS in range(0, 5):
            sel = np.flatnonzero((diagN == N) & (diag2Sz == twoS))
            if len(sel) == 0:
                continue
            hw = _highest_weight(I[:, sel], Sp)
            if hw.shape[1] == 0:
                continue
            h = hw.T @ H @ hw
            e, w = np.linalg.eigh((h + h.T) / 2)
            subs[(N - 2, twoS + 1)] = (e, hw @ w)
    Egs = min(float(e[0]) for e, _ in subs.values())

    def reduced(op_dag: List[np.ndarray]) -> Dict[Tuple[Invar, Invar], np.ndarray]:
        """<I1 || a^dag || I2> of a spin-1/2 creation operator (up, down components)."""
        out = {}
        for (q2, ss2), (_, v2) in subs.items():
            for dss in (+1, -1):
                key1 = (q2 + 1, ss2 + dss)
                if key1 not in subs:
                    continue
                v1 = subs[key1][1]
                S2 = (ss2 - 1) / 2
                if dss > 0:   # m2 = S2; <S2 S2; 1/2 1/2 | S2+1/2 S2+1/2> = 1
                    ket, cg = v2, 1.0
                else:         # m2 = S2 - 1; <S2 S2-1; 1/2 1/2 | S2-1/2 S2-1/2> = -1/sqrt(2 S2 + 1)
                    ket = Sm @ v2
                    ket = ket / np.linalg.norm(ket, axis=0, keepdims=True)
                    cg = -math.sqrt(1.0 / (2 * S2 + 1))
                out[(key1, (q2, ss2))] = (v1.T @ op_dag[0] @ ket) / cg
        return out

    singlets = {"n_d": nd, "n_d^2": nd @ nd, "I": I, "Himp": Himp, "Hhyb": V * hop0, "hop0": hop0}
    order = sorted(subs)
    lines = ["# Input file for NRG Ljubljana", "# symtype \tQS", "#!9",
             "# Number of channels, chain sites, subspaces: ", f"1\t{nmax}\t{len(subs)}",
             f"# SCALE \t{sc!r}", "# Energies (GS energy subtracted, multiplied by 1/SCALE):"]
    for Iv in order:
        e = (subs[Iv][0] - Egs) / sc
        lines += [f"{Iv[0]}\t{Iv[1]}", str(len(e)), "\t".join(repr(float(x)) for x in e)]

    def block(mats: Dict[Tuple[Invar, Invar], np.ndarray]) -> List[str]:
        out = [str(len(mats))]
        for (a, b) in sorted(mats, reverse=True):
            out.append(f"{a[0]}\t{a[1]}\t{b[0]}\t{b[1]}")
            out += ["\t".join(repr(float(x)) for x in row) for row in mats[(a, b)]]
        return out

    lines += ["# Irreducible matrix elements for Wilson chains:", "f 0 0"]
    lines += block(reduced([cd[2], cd[3]]))
    lines += ["# GS energy in absolute units:", "e", repr(float(Egs)),
              "# Irreducible matrix elements for other operators:"]
    for name in ops:
        if name == "A_d":
            lines.append("d" + name)
            lines += block(reduced([cd[0], cd[1]]))
            continue
        if name not in singlets:
            raise ValueError(f"operator {name!r} is not known to the generator")
        O = singlets[name]
        lines.append("s" + name)
        lines += block({(Iv, Iv): subs[Iv][1].T @ O @ subs[Iv][1] for Iv in order})
    lines += ["# Discretization tables:", "z"]
    for tab in (xi, zeta):
        lines.append(str(len(tab) - 1))
        lines += [repr(float(x)) for x in tab]
    return "\n".join(lines) + "\n"


def main(argv=None) -> int:
    """python -m nrgljubljana_b200.datagen --U 1 --delta 0 --Gamma 0.04 --Lambda 2 --Nmax 40
    [--z 1] [--discretization Z] [--ops n_d,A_d] > data"""
    import argparse
    import sys
    ap = argparse.ArgumentParser(description="data file of the QS single-impurity Anderson model")
    ap.add_argument("--U", type=float, required=True)
    ap.add_argument("--delta", type=float, required=True, help="eps_d + U/2")
    ap.add_argument("--Gamma", type=float, required=True)
    ap.add_argument("--Lambda", type=float, default=2.0)
    ap.add_argument("--Nmax", type=int, required=True)
    ap.add_argument("--z", type=float, default=1.0)
    ap.add_argument("--discretization", default="Z", choices=["Z", "C", "Y"])
    ap.add_argument("--ops", default="n_d")
    a = ap.parse_args(argv)
    sys.stdout.write(siam_qs(a.U, a.delta, a.Gamma, a.Lambda, a.Nmax, a.z, a.discretization,
                             [o for o in a.ops.split(",") if o]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
