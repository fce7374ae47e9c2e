"""CPU restatement of an NRG run for symtype QS, one channel -- TEST INFRASTRUCTURE ONLY.

The checker of ``nrgljubljana_b200.nrg_run``: the reference's run loop restated on the
host with LAPACK dsyev and BLAS dgemm through ``oracle.py``. It follows

  docalc0                     c++/core.hpp:251-260
  nrg_loop / iterate          c++/core.hpp:235-248, 286-293
  new_subspaces / structure   c++/core.hpp:42-70, c++/subspaces.hpp:114-121
  hamiltonian + make_matrix   c++/core.hpp:72-88, c++/matrix.hpp:32-78,
                              c++/symmetry/sym-QS-impl.hpp:95-120 with qs-1ch-{offdiag,diag}.dat
  diagonalisations_OpenMP     c++/core.hpp:90-110 (dsyev, one block per thread)
  do_diag                     c++/core.hpp:122-154 (Egs_subtraction, Clusters, truncate_prepare)
  Clusters                    c++/splitting.hpp:24-72
  truncate_prepare            c++/truncation.hpp:14-69
  after_diag                  c++/core.hpp:193-230
  calculate_TD                c++/measurements.hpp:166-186, c++/symmetry/sym-QS-impl.hpp:72-86
  measure_singlet             c++/measurements.hpp:18-30
  recalc_irreduc / recalc_f   c++/symmetry/nrg-recalc-QS.hpp:192-330, c++/recalc.hpp:52-76
  recalc_singlet              c++/symmetry.hpp:185-200, c++/recalc.hpp:82-108

Only ``tests/`` and the CPU-baseline leg of ``bench.py`` may import this module.
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

from . import oracle as O
from nrgljubljana_b200.inputs import SCALE, parse_param, read_data

# QS one-channel tables (c++/symmetry/coefnew/qs/qs-1ch-*.dat)
_IN = [(1, 0), (0, -1), (0, 1), (-1, 0)]
_QN = [(-1, 1), (0, 2), (0, 2), (1, 1)]


def _S(ss):
    return (ss - 1.0) / 2.0


_OFFDIAG = [
    (1, 2, lambda ss: 1),
    (1, 3, lambda ss: 1),
    (2, 4, lambda ss: -(math.sqrt(2) * math.sqrt(_S(ss) / (1 + 2 * _S(ss))))),
    (3, 4, lambda ss: (1 + _S(ss)) / math.sqrt(0.5 + (3 * _S(ss)) / 2. + math.pow(_S(ss), 2))),
]
_DIAG = [(1, 0), (2, 1), (3, 1), (4, 2)]
_SPINUP = [(2, 1, lambda s: 1), (4, 3, lambda s: -math.sqrt(1 - 1 / (2. * (1 + _S(s)))))]
_SPINDOWN = [(3, 1, lambda s: 1), (4, 2, lambda s: math.sqrt(1 + 1 / (2. * _S(s))))]


def _triangle(I, A, Q):
    s1, s2, s3 = I[1], A[1], Q[1]
    return (I[0] == A[0] + Q[0] and abs(s1 - s2) <= s3 - 1 and abs(s2 - s3) <= s1 - 1
            and abs(s3 - s1) <= s2 - 1)


class _Eig:
    def __init__(self, values, vectors=None):
        self.values = values            # relative eigenvalues, ascending
        self.shift = 0.0
        self.corr = values.copy()
        self.vectors = vectors          # rows = eigenvectors (None: identity)
        self.nrstored = len(values)
        self.nrpost = len(values)
        self.U: List[np.ndarray] = []


def run(param_text: str, data_text: str, threads: int = 1) -> Tuple[List[str], List[List[float]], List[str], List[List[float]]]:
    kv = parse_param(param_text)
    Lam = float(kv.get("Lambda", 2.0))
    z = float(kv.get("z", 1.0))
    disc = kv.get("discretization", "Z")
    keep = int(kv.get("keep", 100))
    keepenergy = float(kv.get("keepenergy", -1.0))
    keepmin = int(kv.get("keepmin", 0))
    safeguard = float(kv.get("safeguard", 1e-5))
    safeguardmax = int(kv.get("safeguardmax", 200))
    fixeps = float(kv.get("fixeps", 1e-15))
    betabar = float(kv.get("betabar", 1.0))
    strategy = kv.get("strategy", "kept")
    lastall = kv.get("lastall", "false").lower() == "true"
    rescaled = kv.get("data_has_rescaled_energies", "true").lower() == "true"
    d = read_data(data_text)
    Nmax = d.nmax
    O.blas_threads(1)  # one BLAS thread per block, as diagonalisations_OpenMP runs dsyev

    def scale_of(trueN):
        return SCALE(trueN + 1, Lam, disc, z)

    diag: Dict = {}
    for I, e in sorted(d.subspaces):
        v = e.copy() if rescaled else e / SCALE(0, Lam, disc, z)
        diag[I] = _Eig(v)
    opch = dict(d.opch[0][0])
    ops = {name: {I1: m for (I1, I2), m in mats.items() if I1 == I2}
           for name, (kind, mats) in d.ops.items() if kind in "sg"}

    td_rows, custom_rows = [], []

    def td(trueN, diag):
        f = betabar
        Z = sum(I[1] * sum(math.exp(-f * (x - e.shift)) for x in e.values) for I, e in diag.items())
        E = sum(I[1] * sum(f * (x - e.shift) * math.exp(-f * (x - e.shift)) for x in e.values) for I, e in diag.items())
        E2 = sum(I[1] * sum((f * (x - e.shift)) ** 2 * math.exp(-f * (x - e.shift)) for x in e.values)
                 for I, e in diag.items())
        trSZ = trQ = trQ2 = 0.0
        for I, e in diag.items():
            sumZ = I[1] * sum(math.exp(-f * c) for c in e.corr[:e.nrstored])
            trQ += sumZ * I[0]
            trQ2 += sumZ * I[0] * I[0]
            trSZ += sumZ * (I[1] * I[1] - 1) / 12.
        td_rows.append([scale_of(trueN) / betabar, trSZ / Z, trQ / Z, trQ2 / Z, E / Z, E2 / Z, E2 / Z - (E / Z) ** 2,
                        -math.log(Z), E / Z + math.log(Z)])

    def custom(trueN, diag, ops):
        f = betabar
        Z = sum(I[1] * sum(math.exp(-f * c) for c in e.corr[:e.nrstored]) for I, e in diag.items())
        row = [scale_of(trueN) / betabar]
        for name in sorted(ops):
            tr = 0.0
            for I, e in diag.items():
                m = ops[name][I]
                tr += I[1] * sum(math.exp(-f * e.corr[i]) * m[i, i] for i in range(e.nrstored))
            row.append(tr / Z)
        custom_rows.append(row)

    if kv.get("calc0", "true").lower() == "true":
        td(-1, diag)
        custom(-1, diag, ops)

    for N in range(Nmax):
        last = N == Nmax - 1
        scale = scale_of(N)
        subs = set()
        for I in diag:
            for dlt in _IN:
                J = (I[0] - dlt[0], I[1] - dlt[1])
                if J[1] > 0:
                    subs.add(J)
        structure = {}
        for I in sorted(subs):
            anc = [(I[0] + dl[0], I[1] + dl[1]) for dl in _IN]
            dims = [(diag[a].nrstored if a in diag else 0) if _triangle(I, a, _QN[i]) else 0 for i, a in enumerate(anc)]
            structure[I] = (anc, dims)
        tasks = [I for I in structure if sum(structure[I][1])]
        blocks = []
        for I in tasks:
            anc, dims = structure[I]
            off = np.concatenate([[0], np.cumsum(dims)]).astype(int)
            h = np.zeros((off[-1], off[-1]))
            for i in range(4):
                for n in range(dims[i]):
                    h[off[i] + n, off[i] + n] = math.sqrt(Lam) * diag[anc[i]].corr[n]
            for (i, j, fn) in _OFFDIAG:
                if dims[i - 1] and dims[j - 1]:
                    fs = (fn(I[1]) * d.xi[0][N]) / scale
                    mat = opch[(anc[i - 1], anc[j - 1])]
                    h[off[i - 1]:off[i], off[j - 1]:off[j]] += fs * mat
            for (i, number) in _DIAG:
                for jj in range(off[i - 1], off[i]):
                    h[jj, jj] += d.zeta[0][N + 1] * (number - 1 * 1.0) / scale
            blocks.append(h)
        vals, vecs = O.diag_batch(blocks, nthreads=threads)
        new = {I: _Eig(vals[b], vecs[b]) for b, I in enumerate(tasks)}
        # do_diag
        Egs = min(e.values[0] for e in new.values())
        for e in new.values():
            e.shift = Egs
        energies = sorted(x - e.shift for e in new.values() for x in e.values)
        mapping = {}
        e0, i0, size = energies[0], 0, 1
        for i in range(len(energies)):
            if energies[i] - e0 < fixeps:
                size += 1
            else:
                if size > 1 and any(energies[a] != energies[b] for a in range(i0, i) for b in range(a + 1, i)):
                    for j in range(i0 + 1, i):
                        if energies[j] != energies[i0] and energies[j] not in mapping:
                            mapping[energies[j]] = energies[i0]
                e0, i0, size = energies[i], i, 1
        for e in new.values():
            e.corr = np.array([mapping.get(x - e.shift, x - e.shift) for x in e.values])
        allc = sorted(c for e in new.values() for c in e.corr)
        assert allc[0] == 0.0
        nrkeep = keep if keepenergy <= 0.0 else min(max(1 + sum(1 for c in allc if c <= keepenergy), keepmin), keep)
        extra = 0
        while safeguard > 0.0 and nrkeep < len(allc) and allc[nrkeep] - allc[nrkeep - 1] <= safeguard and extra < safeguardmax:
            nrkeep += 1
            extra += 1
        nrkeep = min(max(nrkeep, 1), len(allc))
        Emax = allc[nrkeep - 1]
        for e in new.values():
            e.nrpost = len(e.values) if (last and lastall) else int(sum(1 for c in e.corr if c <= Emax))
        # after_diag
        td(N, new)
        for I, e in new.items():
            anc, dims = structure[I]
            off = np.concatenate([[0], np.cumsum(dims)]).astype(int)
            e.U = [np.ascontiguousarray(e.vectors[:, off[i]:off[i + 1]]) for i in range(4)]

        def recalc_ops(nrows):
            out = {}
            for name in sorted(ops):
                cold = ops[name]
                cn = {}
                for I, e in new.items():
                    anc, dims = structure[I]
                    k = nrows(e)
                    m = np.zeros((k, k))
                    for i in range(4):
                        a = anc[i]
                        if a[1] <= 0 or a not in cold or k == 0 or dims[i] == 0:
                            continue
                        U = np.ascontiguousarray(e.U[i][:k])
                        Oa = np.ascontiguousarray(cold[a][:dims[i], :dims[i]])
                        O.transform(m, 1.0, U, Oa, U)
                    cn[I] = m
                out[name] = cn
            return out

        if strategy == "all":
            ops = recalc_ops(lambda e: e.nrstored)
            custom(N, new, ops)
        for e in new.values():
            e.nrstored = e.nrpost
        if not last:
            nf = {}
            for Ip, ep in new.items():
                for dq, table in (((1, 1), _SPINUP), ((1, -1), _SPINDOWN)):
                    I1 = (Ip[0] + dq[0], Ip[1] + dq[1])
                    if I1 not in new or not (new[I1].nrstored and ep.nrstored):
                        continue
                    e1 = new[I1]
                    f = np.zeros((e1.nrstored, ep.nrstored))
                    for i1, ip, fn in table:
                        A = np.ascontiguousarray(e1.U[i1 - 1][:e1.nrstored])
                        B = np.ascontiguousarray(ep.U[ip - 1][:ep.nrstored])
                        if A.shape[1] and B.shape[1]:
                            O.product(f, fn(Ip[1]), A, B)
                    nf[(I1, Ip)] = f
            opch = nf
        if strategy == "kept":
            ops = recalc_ops(lambda e: e.nrstored)
            custom(N, new, ops)
        diag = new
    td_fields = ["T", "<Sz^2>", "<Q>", "<Q^2>", "<E>", "<E^2>", "C", "F", "S"]
    return td_fields, td_rows, ["T"] + sorted(ops), custom_rows
