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

The same construction gives the Kondo model of a spin-S impurity coupled to the f0 sites of
one or two channels (``kondo_qs``). Triplet operators (the spin of the d level or of the
impurity) follow nrginit's ireducsigma (nrginit/initial.m:2457-2497): the spherical component
q = S1 - S2 between highest-weight states divided by <S2 S2; 1 q | S1 S1>.

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


# ------------------------------------------------------------------ QS clusters
def _annihilators(nmodes: int) -> List[np.ndarray]:
    """Fermion annihilators of `nmodes` modes, Jordan-Wigner ordered (mode k counts the
    occupied modes below it)."""
    dim = 1 << nmodes
    ops = []
    for k in range(nmodes):
        c = np.zeros((dim, dim))
        for s in range(dim):
            if s >> k & 1:
                sign = -1.0 if bin(s & ((1 << k) - 1)).count("1") % 2 else 1.0
                c[s ^ (1 << k), s] = sign
        ops.append(c)
    return ops


def _spin_matrices(twoS: int) -> Tuple[np.ndarray, np.ndarray]:
    """S_z and S_+ of spin S = twoS/2 in the basis m = S, S-1, ..., -S."""
    S = twoS / 2.0
    m = S - np.arange(twoS + 1)
    Sp = np.zeros((twoS + 1, twoS + 1))
    for k in range(1, twoS + 1):  # S+ |m> = sqrt(S(S+1) - m(m+1)) |m+1>
        Sp[k - 1, k] = math.sqrt(S * (S + 1) - m[k] * (m[k] + 1))
    return np.diag(m), Sp


def _cg(j1: float, m1: float, j2: float, m2: float, J: float, M: float) -> float:
    """Clebsch-Gordan coefficient <j1 m1; j2 m2 | J M> (Condon-Shortley phases), Racah's
    closed formula."""
    if abs(m1 + m2 - M) > 1e-9 or J < abs(j1 - j2) - 1e-9 or J > j1 + j2 + 1e-9:
        return 0.0
    f = math.factorial
    i = lambda x: int(round(x))  # noqa: E731
    pre = math.sqrt((2 * J + 1) * f(i(J + j1 - j2)) * f(i(J - j1 + j2)) * f(i(j1 + j2 - J)) / f(i(j1 + j2 + J + 1)))
    pre *= math.sqrt(f(i(J + M)) * f(i(J - M)) * f(i(j1 - m1)) * f(i(j1 + m1)) * f(i(j2 - m2)) * f(i(j2 + m2)))
    tot = 0.0
    for k in range(0, i(j1 + j2 - J) + 1):
        a = [k, i(j1 + j2 - J - k), i(j1 - m1 - k), i(j2 + m2 - k), i(J - j2 + m1 + k), i(J - j1 - m2 + k)]
        if min(a) < 0:
            continue
        d = 1
        for x in a:
            d *= f(x)
        tot += (-1) ** k / d
    return pre * tot


def _highest_weight(states: np.ndarray, Splus: np.ndarray) -> np.ndarray:
    """Orthonormal basis of the kernel of S+ inside span(states) (columns)."""
    M = Splus @ states
    _, s, vt = np.linalg.svd(M, full_matrices=True)
    rank = int(np.sum(s > 1e-10))
    return states @ vt[rank:].T


class _Cluster:
    """The initial cluster of a QS problem: H, the total charge and spin operators, and
    its multiplets (Q, SS) with the highest-weight eigenvectors of H."""

    def __init__(self, H: np.ndarray, Nop: np.ndarray, Sz: np.ndarray, Sp: np.ndarray, Q0: int):
        self.Sp, self.Sm = Sp, Sp.T
        Nd = np.round(np.diag(Nop)).astype(int)
        Sz2 = np.round(2 * np.diag(Sz)).astype(int)
        eye = np.eye(len(H))
        self.subs: Dict[Invar, Tuple[np.ndarray, np.ndarray]] = {}
        for N in sorted(set(Nd.tolist())):
            for twoS in sorted(set(Sz2.tolist())):
                if twoS < 0:
                    continue
                sel = np.flatnonzero((Nd == N) & (Sz2 == twoS))
                if len(sel) == 0:
                    continue
                hw = _highest_weight(eye[:, sel], Sp)
                if hw.shape[1] == 0:
                    continue
                h = hw.T @ H @ hw
                e, w = np.linalg.eigh((h + h.T) / 2)
                self.subs[(N - Q0, twoS + 1)] = (e, hw @ w)
        self.order = sorted(self.subs)
        self.Egs = min(float(e[0]) for e, _ in self.subs.values())

    def doublet(self, op_dag: Sequence[np.ndarray]) -> Dict[Tuple[Invar, Invar], np.ndarray]:
        """<I1 || a^dag || I2> of a spin-1/2 creation operator (up, down components), with the
        Wigner-Eckart convention <j' m'| T_q |j m> = <j m; 1/2 q | j' m'> <j'||T||j>."""
        out = {}
        for (q2, ss2), (_, v2) in self.subs.items():
            for dss in (+1, -1):
                key1 = (q2 + 1, ss2 + dss)
                if key1 not in self.subs:
                    continue
                v1 = self.subs[key1][1]
                S2 = (ss2 - 1) / 2
                if dss > 0:   # m2 = S2, q = +1/2
                    ket, m2, q = v2, S2, 0.5
                else:         # m2 = S2 - 1, q = +1/2 to reach m1 = S1 = S2 - 1/2
                    ket = self.Sm @ v2
                    ket = ket / np.linalg.norm(ket, axis=0, keepdims=True)
                    m2, q = S2 - 1, 0.5
                S1 = (key1[1] - 1) / 2
                cg = _cg(S2, m2, 0.5, q, S1, S1)
                out[(key1, (q2, ss2))] = (v1.T @ op_dag[0] @ ket) / cg
        return out

    def triplet(self, Sz: np.ndarray, Splus: np.ndarray) -> Dict[Tuple[Invar, Invar], np.ndarray]:
        """<I1 || T || I2> of a spin-1 operator with components S_z, S_+: the spherical
        component q = S1 - S2 between the highest-weight states, divided by
        <S2 S2; 1 q | S1 S1> (1 between two singlets); pairs of equal charge with
        |S1 - S2| <= 1 (nrginit/initial.m:2457-2497)."""
        out = {}
        comp = {0: Sz, 1: -Splus / math.sqrt(2.0), -1: Splus.T / math.sqrt(2.0)}
        for I1 in self.order:
            for I2 in self.order:
                if I1[0] != I2[0] or abs(I1[1] - I2[1]) not in (0, 2):
                    continue
                S1, S2 = (I1[1] - 1) / 2, (I2[1] - 1) / 2
                q = int(round(S1 - S2))
                xa = self.subs[I1][1].T @ comp[q] @ self.subs[I2][1]
                xb = 1.0 if I1[1] == 1 and I2[1] == 1 else _cg(S2, S2, 1.0, q, S1, S1)
                out[(I1, I2)] = xa / xb
        return out

    def singlet(self, O: np.ndarray) -> Dict[Tuple[Invar, Invar], np.ndarray]:
        return {(I, I): self.subs[I][1].T @ O @ self.subs[I][1] for I in self.order}


def _data_text(cl: _Cluster, channels: int, nmax: int, sc: float, fdag: Sequence[Sequence[np.ndarray]],
               ops: Sequence[Tuple[str, str, Dict]], xi: Sequence[np.ndarray], zeta: Sequence[np.ndarray]) -> str:
    """The data file (c++/read-input.hpp): multiplet energies (GS subtracted, / SCALE(0)),
    <||f_ch^dag||> of every channel, the operators (kind letter s/d/t + name) and the
    chain tables (xi of every channel, then zeta of every channel)."""
    lines = ["# Input file for NRG Ljubljana", "# symtype \tQS", "#!9",
             "# Number of channels, chain sites, subspaces: ", f"{channels}\t{nmax}\t{len(cl.subs)}",
             f"# SCALE \t{sc!r}", "# Energies (GS energy subtracted, multiplied by 1/SCALE):"]
    for Iv in cl.order:
        e = (cl.subs[Iv][0] - cl.Egs) / sc
        lines += [f"{Iv[0]}\t{Iv[1]}", str(len(e)), "\t".join(repr(float(x)) for x in e)]

    def block(mats: Dict[Tuple[Invar, Invar], np.ndarray]) -> List[str]:
        out = [str(len(mats))]
        for (a, b) in sorted(mats, reverse=True):
            out.append(f"{a[0]}\t{a[1]}\t{b[0]}\t{b[1]}")
            out += ["\t".join(repr(float(x)) for x in row) for row in mats[(a, b)]]
        return out

    lines.append("# Irreducible matrix elements for Wilson chains:")
    for ch in range(channels):
        lines.append(f"f {ch} 0")
        lines += block(cl.doublet(fdag[ch]))
    lines += ["# GS energy in absolute units:", "e", repr(float(cl.Egs)),
              "# Irreducible matrix elements for other operators:"]
    for kind, name, mats in ops:
        lines.append(kind + name)
        lines += block(mats)
    lines += ["# Discretization tables:", "z"]
    for tab in list(xi) + list(zeta):
        lines.append(str(len(tab) - 1))
        lines += [repr(float(x)) for x in tab]
    return "\n".join(lines) + "\n"


def _spin_ops(c: Sequence[np.ndarray], up: int, dn: int) -> Tuple[np.ndarray, np.ndarray]:
    """S_z and S_+ of the electron in modes (up, dn)."""
    cd = [m.T for m in c]
    return 0.5 * (cd[up] @ c[up] - cd[dn] @ c[dn]), cd[up] @ c[dn]


def siam_qs(U: float, delta: float, Gamma: float, Lambda: float, nmax: int, z: float = 1.0,
            discretization: str = "Z", ops: Sequence[str] = ("n_d",), xi=None, zeta=None) -> str:
    """The ``data`` file of the QS single-impurity Anderson model (one channel, flat band).

    delta = eps_d + U/2. Operators: singlets n_d, n_d^2, I, Himp, Hhyb, hop0, the doublet A_d
    (d^dag) and the triplet sigma_d (the spin of the d level)."""
    if xi is None or zeta is None:
        xi, zeta = wilson_chain(Lambda, nmax, z, discretization)
    # modes 0: d up, 1: d down, 2: f0 up, 3: f0 down
    c = _annihilators(4)
    cd = [m.T for m in c]
    n = [cd[k] @ c[k] for k in range(4)]
    nd = n[0] + n[1]
    nf = n[2] + n[3]
    I = np.eye(16)
    V = math.sqrt(2.0 * Gamma * gamma_A(Lambda, discretization) / math.pi)
    hop0 = sum(cd[2 + s] @ c[s] + cd[s] @ c[2 + s] for s in (0, 1))
    Himp = delta * nd + U / 2 * (nd - I) @ (nd - I)
    H = Himp + V * hop0 + zeta[0] * (nf - I)
    Szd, Spd = _spin_ops(c, 0, 1)
    Szf, Spf = _spin_ops(c, 2, 3)
    cl = _Cluster(H, nd + nf, Szd + Szf, Spd + Spf, Q0=2)
    singlets = {"n_d": nd, "n_d^2": nd @ nd, "I": I, "Himp": Himp, "Hhyb": V * hop0, "hop0": hop0}
    out = []
    for name in ops:
        if name == "A_d":
            out.append(("d", name, cl.doublet([cd[0], cd[1]])))
        elif name == "sigma_d":
            out.append(("t", name, cl.triplet(Szd, Spd)))
        elif name in singlets:
            out.append(("s", name, cl.singlet(singlets[name])))
        else:
            raise ValueError(f"operator {name!r} is not known to the generator")
    return _data_text(cl, 1, nmax, scale0(Lambda, z, discretization), [[cd[2], cd[3]]], out, [xi], [zeta])


def kondo_qs(J: Sequence[float], spin: float, Lambda: float, nmax: int, z: float = 1.0, discretization: str = "Z",
             ops: Sequence[str] = (), xi=None, zeta=None) -> str:
    """The ``data`` file of the QS Kondo model with len(J) channels (one or two) coupled to an
    impurity spin `spin`: H = sum_ch J[ch] S . s_f0(ch) + zeta_0 (n_f0(ch) - 1), flat band
    (the model of the reference's test/c++sym_all/test300_QS_ref/kondo.m; for spin 1/2 the
    same spectrum as the projected model ONE/KONDO, nrginit/models.m:822-834).

    Q = N - channels (N electrons on the f0 sites); SS = 2 S_tot + 1. Operators: singlets
    q_f = n_f0(0) - 1, q_f^2, n_f (f0 of channel 0), S.s_f (S . s_f0(0)), the triplets S_imp
    (the impurity spin) and sigma_f (the spin of f0 of channel 0)."""
    channels = len(J)
    if channels not in (1, 2):
        raise ValueError("one or two channels")
    twoS = int(round(2 * spin))
    if twoS < 1 or abs(twoS - 2 * spin) > 1e-12:
        raise ValueError("spin must be a positive multiple of 1/2")
    if xi is None or zeta is None:
        xi, zeta = wilson_chain(Lambda, nmax, z, discretization)
    xis = [xi] * channels
    zetas = [zeta] * channels
    # modes 2ch: f0 up, 2ch + 1: f0 down of channel ch; the impurity spin is the slower index
    nm = 2 * channels
    c0 = _annihilators(nm)
    If = np.eye(1 << nm)
    Szi0, Spi0 = _spin_matrices(twoS)
    Ii = np.eye(twoS + 1)
    c = [np.kron(Ii, m) for m in c0]
    cd = [m.T for m in c]
    Szi, Spi = np.kron(Szi0, If), np.kron(Spi0, If)
    I = np.eye(len(c[0]))
    nf = [cd[2 * ch] @ c[2 * ch] + cd[2 * ch + 1] @ c[2 * ch + 1] for ch in range(channels)]
    sz, sp = zip(*[_spin_ops(c, 2 * ch, 2 * ch + 1) for ch in range(channels)])
    H = np.zeros_like(I)
    SS = []
    for ch in range(channels):
        ss = Szi @ sz[ch] + 0.5 * (Spi @ sp[ch].T + Spi.T @ sp[ch])
        SS.append(ss)
        H = H + J[ch] * ss + zetas[ch][0] * (nf[ch] - I)
    cl = _Cluster(H, sum(nf), Szi + sum(sz), Spi + sum(sp), Q0=channels)
    singlets = {"q_f": nf[0] - I, "q_f^2": (nf[0] - I) @ (nf[0] - I), "n_f": nf[0], "S.s_f": SS[0]}
    out = []
    for name in ops:
        if name == "S_imp":
            out.append(("t", name, cl.triplet(Szi, Spi)))
        elif name == "sigma_f":
            out.append(("t", name, cl.triplet(sz[0], sp[0])))
        elif name in singlets:
            out.append(("s", name, cl.singlet(singlets[name])))
        else:
            raise ValueError(f"operator {name!r} is not known to the generator")
    fdag = [[cd[2 * ch], cd[2 * ch + 1]] for ch in range(channels)]
    return _data_text(cl, channels, nmax, scale0(Lambda, z, discretization), fdag, out, xis, zetas)


def main(argv=None) -> int:
    """python -m nrgljubljana_b200.datagen siam --U 1 --delta 0 --Gamma 0.04 --Lambda 2 --Nmax 40
    [--z 1] [--discretization Z] [--ops n_d,A_d] > data
    python -m nrgljubljana_b200.datagen kondo --J 0.2,0.2 --spin 1 --Lambda 3 --Nmax 50 [--ops S_imp] > data"""
    import argparse
    import sys
    ap = argparse.ArgumentParser(description="data file of a QS impurity model")
    ap.add_argument("model", choices=["siam", "kondo"])
    ap.add_argument("--U", type=float, default=1.0)
    ap.add_argument("--delta", type=float, default=0.0, help="eps_d + U/2")
    ap.add_argument("--Gamma", type=float, default=0.04)
    ap.add_argument("--J", default="0.2", help="Kondo couplings, one per channel")
    ap.add_argument("--spin", type=float, default=0.5, help="impurity spin of the Kondo model")
    ap.add_argument("--Lambda", type=float, default=2.0)
    ap.add_argument("--Nmax", type=int, required=True)
    ap.add_argument("--z", type=float, default=1.0)
    ap.add_argument("--discretization", default="Z", choices=["Z", "C", "Y"])
    ap.add_argument("--ops", default="")
    a = ap.parse_args(argv)
    ops = [o for o in a.ops.split(",") if o]
    if a.model == "siam":
        sys.stdout.write(siam_qs(a.U, a.delta, a.Gamma, a.Lambda, a.Nmax, a.z, a.discretization, ops or ["n_d"]))
    else:
        sys.stdout.write(kondo_qs([float(x) for x in a.J.split(",")], a.spin, a.Lambda, a.Nmax, a.z,
                                  a.discretization, ops))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
