"""CPU restatement of an NRG run for symtype QS, one or two channels -- TEST INFRASTRUCTURE ONLY.

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
  recalc_global (QS, 2 ch.)   c++/symmetry/nrg-recalc-QS.hpp:680-740, c++/recalc.hpp:111-122,
                              qs-2ch-{q1,q2,qdiff,qtot}.dat
  recalc_doublet (QS)         c++/symmetry/nrg-recalc-QS.hpp:32-117, qs-1ch-doublet{p,m}.dat
  DM-NRG                      init_rho, cdmI, calc_densitymatrix(_iterN) c++/dmnrg.hpp:43-112;
                              Algo_DMNRG c++/algo_DMNRG.hpp:29-52; BaseSpectrum::calc c++/algo.hpp:55-67;
                              mergeNN2half, windowfunction, continuous c++/spectrum.hpp:81-196;
                              Bins c++/bins.hpp:61-185; BR_NEW c++/spectral.hpp:42-70
  FDM                         c++/dmnrg.hpp:146-217; Algo_FDMgt/ls c++/algo_FDM.hpp:30-151;
                              Algo_FDMmats c++/algo_FDM.hpp:153-217, GFMatsubara c++/spectrum.hpp:212-227,
                              Matsubara c++/matsubara.hpp:19-58;
                              calc_ZnD, fdm_thermodynamics c++/measurements.hpp:60-163
  CFS, FT                     Algo_CFSgt/ls c++/algo_CFS.hpp:28-105; Algo_FT c++/algo_FT.hpp:28-48;
                              calc_Z c++/measurements.hpp:189-191
  output                      savebins c++/spectrum.hpp:146-170; Annotated::dump
                              c++/output.hpp:77-125; dump_energies c++/output.hpp:157-161

Only ``tests/`` and the CPU-baseline leg of ``bench.py`` may import this module.
"""
from __future__ import annotations

import math
from fractions import Fraction
from typing import Dict, List, Tuple

import numpy as np

from . import oracle as O
from nrgljubljana_b200.inputs import SCALE, parse_param, read_data

# The QS coefficient tables (In, QN, the diagonal / off-diagonal factors and the <||f||>
# recalculation rows of c++/symmetry/coefnew/qs/qs-{1,2}ch-*.dat) are data of the symmetry,
# shared with the product (nrgljubljana_b200.qs); they are pinned by the reference's
# regression outputs through both implementations.
from nrgljubljana_b200 import qs as _qs


def _S(ss):
    return (ss - 1.0) / 2.0


# doublet recalculation, Ip = (q1 - 1, ss1 + 1) and (q1 - 1, ss1 - 1): rows (i1, ip, factor(ss1))
_DOUBLETP = [(1, 1, lambda s: 1), (2, 2, lambda s: (-2 * math.sqrt(_S(s) * (1 + _S(s)))) / (1 + 2 * _S(s))),
             (3, 2, lambda s: 1 / (1 + 2 * _S(s))), (3, 3, lambda s: -1), (4, 4, lambda s: 1)]
_DOUBLETM = [(1, 1, lambda s: 1), (2, 2, lambda s: -1), (2, 3, lambda s: 1 / (-1 - 2 * _S(s))),
             (3, 3, lambda s: (-2 * (1 + _S(s))) / math.sqrt(5 + 1 / _S(s) + 8 * _S(s) + 4 * math.pow(_S(s), 2))),
             (4, 4, lambda s: 1)]


def _specdens_factor(Ip, I1):
    """SymmetryQS::specdens_factor (c++/symmetry/sym-QS-impl.hpp:64-70)."""
    return _S(Ip[1]) + 1.0 if I1[1] == Ip[1] + 1 else _S(Ip[1])


def _BR_NEW(e, ept, alpha, omega0):
    """c++/spectral.hpp:42-70."""
    part_l = 0.0
    if not ((e < 0.0 and ept > 0.0) or (e > 0.0 and ept < 0.0) or ept == 0.0):
        gamma = alpha / 4.0
        part_l = math.exp(-math.pow(math.log(e / ept) / alpha - gamma, 2)) / (alpha * abs(e) * math.sqrt(math.pi))
    if abs(e) > omega0:
        return part_l
    BR_h = math.exp(-math.pow(math.log(abs(e) / omega0) / alpha, 2))
    BR_G = math.exp(-math.pow((e - ept) / omega0, 2)) / (omega0 * math.sqrt(math.pi))
    return part_l * BR_h + BR_G * (1.0 - BR_h)


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


def run(param_text: str, data_text: str, threads: int = 1, spectra: dict = None, fdm_out: dict = None,
        bins_out: dict = None, annotated_out: list = None, annotated_entries: list = None,
        energies_out: list = None, subspaces_out: list = None) -> Tuple[List[str], List[List[float]], List[str], List[List[float]]]:
    """td and custom rows of the run; with a `spectra` dict, also the spectra of the specs,
    specd and spect pairs for the algorithms dmnrg, fdm, fdmgt, fdmls that are switched on
    (file stem, e.g. spec_DMNRG_dens_A_d-A_d -> array of (E, A(E)) rows as written to that
    .dat file); with an `fdm_out` dict and an FDM flag, also fdm_out["tdfdm"] (fields, row)
    and, with fdmexpv, fdm_out["customfdm"] (fields, row); with a `bins_out` dict and a
    `spectra` dict, also the trimmed raw bins of every spectrum as savebins writes them
    (SpectrumRealFreq::savebins, c++/spectrum.hpp:146-170): rows (E, Re w), or (E, Re w, Im w)
    with reim=true, the positive energies ascending, then -|E| by ascending |E|; with an
    `annotated_out` list, the lines of annotated.dat (Annotated::dump, c++/output.hpp:77-125)
    for dumpannotated > 0 (and, in `annotated_entries`, each step's (energy, subspace) pairs
    with its scale and total energy, the formatter's input); with an `energies_out` list and
    dumpenergies=true, the text of energies.nrg (Output::dump_energies, c++/output.hpp:157-161);
    with a `subspaces_out` list and dumpsubspaces=true, the lines of subspaces.dat
    (Store::dump_subspaces, c++/store.hpp:75-84)."""
    kv = parse_param(param_text)
    Lam = float(kv.get("Lambda", 2.0))
    z = float(kv.get("z", 1.0))
    disc = kv.get("discretization", "Z")
    brs = float(kv.get("bandrescale", 1.0))  # Params::SCALE multiplies by bandrescale (c++/params.hpp:632)
    keep = int(kv.get("keep", 100))
    keepenergy = float(kv.get("keepenergy", -1.0))
    keepmin = int(kv.get("keepmin", 0))
    safeguard = float(kv.get("safeguard", 1e-5))
    safeguardmax = int(kv.get("safeguardmax", 200))
    fixeps = float(kv.get("fixeps", 1e-15))
    betabar = float(kv.get("betabar", 1.0))
    strategy = kv.get("strategy", "kept")
    flag = lambda k: kv.get(k, "false").lower() == "true"  # noqa: E731
    # Params::cfs_flags, fdm_flags, keep_all_states_in_last_step (c++/params.hpp:534-539)
    cfs_flags = any(flag(k) for k in ("cfs", "cfsgt", "cfsls"))
    fdm_flags = any(flag(k) for k in ("fdm", "fdmgt", "fdmls", "fdmmats", "fdmexpv"))
    lastall = flag("lastall") or ((cfs_flags or fdm_flags) and not flag("lastalloverride"))
    rescaled = kv.get("data_has_rescaled_energies", "true").lower() == "true"
    d = read_data(data_text)
    Nmax = d.nmax
    T = _qs.tables(d.channels)
    _IN, _QN, C = T.IN, T.QN, T.COMBS
    O.blas_threads(1)  # one BLAS thread per block, as diagonalisations_OpenMP runs dsyev

    def scale_of(trueN):
        return SCALE(trueN + 1, Lam, disc, z, brs)

    diag: Dict = {}
    for I, e in sorted(d.subspaces):
        v = e.copy() if rescaled else e / SCALE(0, Lam, disc, z, brs)
        diag[I] = _Eig(v)
    opch = [dict(d.opch[ch][0]) for ch in range(d.channels)]
    ops = {name: {I1: m for (I1, I2), m in mats.items() if I1 == I2}
           for name, (kind, mats) in d.ops.items() if kind in "sg"}
    gops = {name for name, (kind, _) in d.ops.items() if kind == "g"}
    if not gops <= set(T.GLOBAL):
        raise ValueError(f"global operators {sorted(gops - set(T.GLOBAL))}: not in recalc_global")

    def singlet_order(names):
        """Singlets, then global operators, each by name (c++/output.hpp:121-127)."""
        return sorted(set(names) - gops) + sorted(set(names) & gops)
    # spectral algorithms (c++/oprecalc.hpp:107-132) and the FDM flags (c++/params.hpp:535-541)
    algos = [a for a, k in (("DMNRG", "dmnrg"), ("DMNRGmats", "dmnrgmats"), ("FDM", "fdm"), ("FDMgt", "fdmgt"),
                            ("FDMls", "fdmls"), ("FDMmats", "fdmmats"), ("FTmats", "finitemats"),
                            ("CFS", "cfs"), ("CFSgt", "cfsgt"), ("CFSls", "cfsls"), ("FT", "finite")) if flag(k)]
    dm = spectra is not None and bool(algos)
    fdm_needed = fdm_flags and (spectra is not None or fdm_out is not None)
    total_energy = d.gs_energy  # Stats::total_energy (c++/stats.hpp:60-71)

    def pairs(key):
        return [tuple(t.split("-", 1)) for t in kv.get(key, "").split()] if dm else []
    # (file prefix, kind, op1, op2): correlators of singlets, spectral functions of doublets,
    # dynamic spin susceptibilities of triplets (c++/oprecalc.hpp:160-195)
    specs = [("corr", "s") + pr for pr in pairs("specs")] + [("spec", "d") + pr for pr in pairs("specd")] + \
        [("spin", "t") + pr for pr in pairs("spect")]
    dops = {name: dict(d.ops[name][1]) for name in sorted({x for sp in specs if sp[1] == "d" for x in sp[2:]})}
    tops = {name: dict(d.ops[name][1]) for name in sorted({x for sp in specs if sp[1] == "t" for x in sp[2:]})}
    for sp in specs:
        if sp[1] == "s" and not set(sp[2:]) <= set(ops):
            raise ValueError(f"specs names an operator that is not a singlet of the data file: {sp}")
    steps = []  # per step: subspaces, structure, operators of the spectra (DM-NRG)

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
        for name in singlet_order(ops):
            tr = 0.0
            for I, e in diag.items():
                m = ops[name][I]
                tr += I[1] * sum(math.exp(-f * e.corr[i]) * m[i, i] for i in range(e.nrstored))
            row.append(tr / Z)
        custom_rows.append(row)

    dumpannotated = int(kv.get("dumpannotated", 0))

    def dump_energies(diag, trueN):
        """Output::dump_energies with DiagInfo::dump_energies (c++/eigen.hpp:349-352): per call
        a header with the step index max(N, 0), then every subspace in order with its raw
        eigenvalues (all_rel: the ground-state shift is not subtracted), printed as a C++
        stream prints a vector of doubles."""
        if energies_out is None or not flag("dumpenergies"):
            return
        text = "\n===== Iteration number: %d\n" % max(trueN, 0)
        for I in sorted(diag):
            e = diag[I]
            text += "Subspace: %d %d\n" % I + "".join("%g " % x for x in e.values) + "\n"
        energies_out.append(text)

    def annotate(diag, scale):
        """Annotated::dump (c++/output.hpp:77-125): the lowest dumpannotated energies of all
        computed states (extended over a cluster at the cut), grouped by degeneracy with
        my_fcmp (c++/numerics.hpp:107-114) at grouptol."""
        if annotated_out is None or dumpannotated <= 0:
            return
        tol = float(kv.get("grouptol", 1e-6))
        prec = int(kv.get("dumpprecision", 8))
        groups = kv.get("dumpgroups", "true").lower() == "true"
        scaled = kv.get("dumpscaled", "true").lower() == "true"
        absolute = kv.get("dumpabs", "false").lower() == "true"

        def cmp(x, y):
            if (x == 0.0 and y == 0.0) or (abs(x) < tol and abs(y) < tol) or abs(x - y) < tol * (abs(x) + abs(y)):
                return 0
            return 1 if x > y else -1
        if annotated_entries is not None:
            annotated_entries.append(([(x - e.shift, I) for I, e in diag.items() for x in e.values], scale, total_energy))
        lst = sorted((x - e.shift, I) for I, e in diag.items() for x in e.values)
        n = min(len(lst), dumpannotated)
        while n < len(lst) - 1 and cmp(lst[n][0], lst[n - 1][0]) == 0:
            n += 1

        def num(x):
            return "%.*g" % (prec, x * (1.0 if scaled else scale) + (total_energy if absolute else 0.0))
        if groups:
            i = 0
            while i < n:
                e0 = lst[i][0]
                names, deg = [], 0
                while i < n and cmp(lst[i][0], e0) == 0:
                    names.append("%d %d" % lst[i][1])
                    deg += lst[i][1][1]  # multiplicity of a QS subspace: 2S+1 = SS
                    i += 1
                annotated_out.append(num(e0) + "".join(" (%s)" % q for q in sorted(names)) + " [%d]" % deg)
        else:
            annotated_out.extend("%s %d %d" % (num(e), I[0], I[1]) for e, I in lst[:n])
        annotated_out.append("")

    init_spec = None
    if kv.get("calc0", "true").lower() == "true":
        dump_energies(diag, -1)
        annotate(diag, SCALE(0, Lam, disc, z, brs))
        td(-1, diag)
        custom(-1, diag, ops)
        # docalc0 runs the first run's spectral algorithms on the initial cluster too
        # (c++/core.hpp:251-260): its eigenvalues with shift 0 and scale SCALE(Ninit), every
        # state kept, the operators as read (c++/eigen.hpp:219-226, 314)
        init_spec = (SCALE(0, Lam, disc, z, brs), {I: e.values.copy() for I, e in diag.items()},
                     {"s": {name: {(I, I): m for I, m in ops[name].items()} for name in ops},
                      "d": {name: dict(m) for name, m in dops.items()}, "t": {name: dict(m) for name, m in tops.items()}})

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
            for i in range(C):
                for n in range(dims[i]):
                    h[off[i] + n, off[i] + n] = math.sqrt(Lam) * diag[anc[i]].corr[n]
            for (i, j, ch, fn) in T.OFFDIAG:
                if dims[i - 1] and dims[j - 1]:
                    fs = (_qs.ieee(fn, I[1]) * d.xi[ch][N]) / scale
                    mat = opch[ch][(anc[i - 1], anc[j - 1])]
                    if i > j:
                        h[off[j - 1]:off[j], off[i - 1]:off[i]] += fs * mat.T
                    else:
                        h[off[i - 1]:off[i], off[j - 1]:off[j]] += fs * mat
            for (i, ch, number) in T.DIAG:
                for jj in range(off[i - 1], off[i]):
                    h[jj, jj] += d.zeta[ch][N + 1] * (number - 1 * 1.0) / scale
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
        if subspaces_out is not None and flag("dumpsubspaces"):  # the Store of the run, dumped after it
            subspaces_out.append("Iteration %d" % N)
            subspaces_out.append("len_dm=%d" % len(new))
            for I in sorted(new):
                subspaces_out.append("I=%d %d kept=%d total=%d" % (I[0], I[1], new[I].nrpost, len(new[I].values)))
            subspaces_out.append("")
        # after_diag
        total_energy += Egs * scale  # Stats::update (c++/stats.hpp:65-71)
        dump_energies(new, N)
        annotate(new, scale)
        td(N, new)
        ops_prev = ops
        for I, e in new.items():
            anc, dims = structure[I]
            off = np.concatenate([[0], np.cumsum(dims)]).astype(int)
            e.U = [np.ascontiguousarray(e.vectors[:, off[i]:off[i + 1]]) for i in range(C)]

        def recalc_ops(nrows, names=None):
            out = {}
            for name in sorted(ops_prev if names is None else names):
                cold = ops_prev[name]
                cn = {}
                for I, e in new.items():
                    anc, dims = structure[I]
                    k = nrows(e)
                    m = np.zeros((k, k))
                    for i in range(C):
                        a = anc[i]
                        if a[1] <= 0 or a not in cold or k == 0 or dims[i] == 0:
                            continue
                        U = np.ascontiguousarray(e.U[i][:k])
                        Oa = np.ascontiguousarray(cold[a][:dims[i], :dims[i]])
                        O.transform(m, 1.0, U, Oa, U)
                    # recalc_global: the charge of the added site, product(m, value, U_i1, U_ip)
                    for i1, ip, _, value in (T.GLOBAL[name] if name in gops else ()):
                        if k and dims[i1 - 1] and dims[ip - 1]:
                            O.product(m, float(value), np.ascontiguousarray(e.U[i1 - 1][:k]),
                                      np.ascontiguousarray(e.U[ip - 1][:k]))
                    cn[I] = m
                out[name] = cn
            return out

        if strategy == "all":
            ops = recalc_ops(lambda e: e.nrstored)
            custom(N, new, ops)
        for e in new.values():
            e.nrstored = e.nrpost
        if not last:
            nf = [dict() for _ in range(d.channels)]
            for Ip, ep in new.items():
                for dq, ch, table in T.RECALC_F:
                    I1 = (Ip[0] + dq[0], Ip[1] + dq[1])
                    if I1 not in new or not (new[I1].nrstored and ep.nrstored):
                        continue
                    e1 = new[I1]
                    f = np.zeros((e1.nrstored, ep.nrstored))
                    for i1, ip, fn in table:
                        A = np.ascontiguousarray(e1.U[i1 - 1][:e1.nrstored])
                        B = np.ascontiguousarray(ep.U[ip - 1][:ep.nrstored])
                        if A.shape[1] and B.shape[1]:
                            O.product(f, _qs.ieee(fn, Ip[1]), A, B)
                    nf[ch][(I1, Ip)] = f
            opch = nf
        if strategy == "kept":
            ops = recalc_ops(lambda e: e.nrstored)
            custom(N, new, ops)
        if dm or fdm_needed:
            # The DMNRG run recalculates the operators of the spectra over all states when a CFS
            # or FDM flag is set (do_recalc_all, c++/params.hpp:542-547), else over the kept ones.
            nrows = (lambda e: len(e.values)) if (cfs_flags or fdm_flags) else (lambda e: e.nrstored)  # noqa: E731

            def recalc_tensor(cold, tables, factor):
                """recalc_general (c++/recalc.hpp:82-108) over the pairs Ip = I1 + dq."""
                cn = {}
                for I1, e1 in new.items():
                    for dq, table in tables:
                        Ip = (I1[0] + dq[0], I1[1] + dq[1])
                        if Ip not in new or not (nrows(e1) and nrows(new[Ip])):
                            continue
                        ep = new[Ip]
                        r1, rp = nrows(e1), nrows(ep)
                        m = np.zeros((r1, rp))
                        anc1, dims1 = structure[I1]
                        ancp, dimsp = structure[Ip]
                        for i1, ip, fn in table:
                            IN1, INp = anc1[i1 - 1], ancp[ip - 1]
                            if IN1[1] <= 0 or INp[1] <= 0 or (IN1, INp) not in cold:
                                continue
                            if dims1[i1 - 1] == 0 or dimsp[ip - 1] == 0:
                                continue
                            A = np.ascontiguousarray(e1.U[i1 - 1][:r1])
                            B = np.ascontiguousarray(ep.U[ip - 1][:rp])
                            Oa = np.ascontiguousarray(cold[(IN1, INp)][:dims1[i1 - 1], :dimsp[ip - 1]])
                            O.transform(m, factor(fn, I1[1]), A, Oa, B)
                        cn[(I1, Ip)] = m
                return cn
            # recalc_doublet (nrg-recalc-QS.hpp:32-117), recalc_triplet (495-640)
            if d.channels == 1:
                dtab, dfac = (((-1, 1), _DOUBLETP), ((-1, -1), _DOUBLETM)), (lambda fn, ss: fn(ss))
            else:
                dtab, dfac = T.DOUBLET, T.doublet_factor
            dops = {name: recalc_tensor(cold, dtab, dfac) for name, cold in dops.items()}
            tops = {name: recalc_tensor(cold, T.TRIPLET, _qs.triplet_factor) for name, cold in tops.items()}
            snames = {x for sp in specs if sp[1] == "s" for x in sp[2:]}
            if cfs_flags or fdm_flags:
                snames |= set(ops) if (fdm_out is not None and flag("fdmexpv")) else set()
                sops = recalc_ops(nrows, snames)
            else:
                sops = {name: ops[name] for name in snames}
            sops = {name: {(I, I): m for I, m in mats.items()} for name, mats in sops.items()}
            steps.append((N, scale, new, structure, {"s": sops, "d": dops, "t": tops}, total_energy))
        diag = new
    if (dm or fdm_needed) and steps:
        _dm_outputs(kv, steps, Lam, disc, z, Nmax, specs, algos if dm else [], spectra, fdm_out if fdm_flags else None,
                    total_energy, C, singlet_order(ops), bins_out=bins_out, init_spec=init_spec)
    td_fields = ["T", "<Sz^2>", "<Q>", "<Q^2>", "<E>", "<E^2>", "C", "F", "S"]
    return td_fields, td_rows, ["T"] + singlet_order(ops), custom_rows


def _exact_sum(values) -> Fraction:
    """The exact sum of doubles (dyadic rationals) as a Fraction."""
    ratios = [float(v).as_integer_ratio() for v in values]
    if not ratios:
        return Fraction(0)
    D = max(d for _, d in ratios)
    return Fraction(sum(n * (D // d) for n, d in ratios), D)


def _exact_dot(a, b) -> Fraction:
    """The exact sum of the products a[i] * b[i] of doubles."""
    ra = [float(v).as_integer_ratio() for v in a]
    rb = [float(v).as_integer_ratio() for v in b]
    if not ra:
        return Fraction(0)
    terms = [(n1 * n2, d1 * d2) for (n1, d1), (n2, d2) in zip(ra, rb)]
    D = max(d for _, d in terms)
    return Fraction(sum(n * (D // d) for n, d in terms), D)


def _fdm_weights(steps, T, GS, combs):
    """calc_ZnD and fdm_thermodynamics (c++/measurements.hpp:60-163). The reference sums in
    400-bit GMP; exact rational sums of the same double terms stand in for it. Returns the
    per-step wn, wnfactor, ZnDN (double) and the tdfdm row (T, E, C, F, S)."""
    Nend = len(steps)
    ZG, ZN = [], []
    for k, (N, scale, diagN, _, _, Tshift) in enumerate(steps):
        last = k == Nend - 1
        g, n = [], []
        for I, e in diagN.items():
            lo = 0 if last else e.nrpost      # Sub::all(), c++/store.hpp:26-31: the D states
            for x in e.values[lo:]:
                absz = (x - e.shift) * scale  # Values::abs_zero, abs_T, abs_G (c++/eigen.hpp:42-47)
                absg = (absz + Tshift) - GS
                g.append(I[1] * math.exp(-absg / T))
                n.append(I[1] * math.exp(-absz / T))
        ZG.append(_exact_sum(g))
        ZN.append(_exact_sum(n))
    ZZG = sum(ZG[k] * combs ** (Nend - k - 1) for k in range(Nend))
    ZZGd = float(ZZG)
    wnfactor = [math.pow(combs, Nend - k - 1) / ZZGd for k in range(Nend)]
    wn = [wnfactor[k] * float(ZG[k]) for k in range(Nend)]
    assert abs(sum(wn) - 1.0) < 1e-12, sum(wn)  # the sum rule, num_equal(sumwn, 1.0)
    E = Fraction(0)
    E2 = Fraction(0)
    for k, (N, scale, diagN, _, _, Tshift) in enumerate(steps):
        if not wn[k] > 1e-16:
            continue
        last = k == Nend - 1
        d, e1, e2 = [], [], []
        for I, e in diagN.items():
            lo = 0 if last else e.nrpost
            for x in e.values[lo:]:
                absz = (x - e.shift) * scale
                absT = absz + Tshift
                d.append(wn[k] * I[1] * math.exp(-absz / T))
                e1.append(absT)
        sd = _exact_dot(d, e1)
        sd2 = sum((Fraction(w) * Fraction(x) * Fraction(x) for w, x in zip(d, e1)), Fraction(0))
        E += sd / ZN[k]
        E2 += sd2 / ZN[k]
    E_fdm = float(E)
    C_fdm = float(E2 - E * E) / math.pow(T, 2)
    F_fdm = -math.log(ZZGd) * T + GS
    S_fdm = (E_fdm - F_fdm) / T
    return wn, wnfactor, [float(z) for z in ZN], [T, E_fdm, C_fdm, F_fdm, S_fdm]


def cfs_terms(last, Ei, ki, Ej, kj, o1, o2, rho_i, rho_j, sign, T, Zft):
    """The (energy, weight) terms of Algo_CFSgt::calc and Algo_CFSls::calc (c++/algo_CFS.hpp:
    28-53, 80-105) for one pair, in the reference's loop order, with Ip = Ii and I1 = Ij:
    o1, o2 = op(Ij, Ii) (r1 in Ij rows, rp in Ii columns) over all states; Ei, Ej the abs_zero
    energies of all states; ki, kj the kept states; rho_i, rho_j the DM-NRG density matrices
    (kept x kept) of Ii, Ij; Zft the last step's kept-state partition function. Returns
    {"gt": (E, w), "ls": (E, w)} before the factor ff(Ii, Ij)."""
    if last:  # i-term, Eq. (11): r1 in kept(I1), rp in kept(Ip)
        E = (Ej[:kj, None] - Ei[None, :ki]).ravel()
        base = o1[:kj, :ki] * o2[:kj, :ki]
        return {"gt": (E, (base * np.exp(-Ei[None, :ki] / T) / Zft).ravel()),
                "ls": (E, (base * np.exp(-Ej[:kj, None] / T) * (-sign) / Zft).ravel())}
    # ii-term, Eq. (15): rk in kept(I1), rl in discarded(Ip);
    # op1_rho = prod_adj_fit_left(op1, rho(I1)) (c++/numerics.hpp:310-316)
    o1rho = o1[:kj, :].T @ rho_j
    E_gt = (Ej[:kj, None] - Ei[None, ki:]).ravel()
    w_gt = (o1rho[ki:, :].T * o2[:kj, ki:]).ravel()
    # iii-term, Eq. (16): rl in discarded(I1), rk in kept(Ip);
    # op2_rho = prod_fit_left(op2, rho(Ip)) (c++/numerics.hpp:285-291)
    o2rho = o2[:, :ki] @ rho_i
    E_ls = (Ej[kj:, None] - Ei[None, :ki]).ravel()
    w_ls = (o1[kj:, :ki] * o2rho[kj:, :] * (-sign)).ravel()
    return {"gt": (E_gt, w_gt), "ls": (E_ls, w_ls)}


def ft_terms(Ei, Ej, o1, o2, sign, T, Z):
    """The (energy, weight) terms of Algo_FT::calc (c++/algo_FT.hpp:28-43) for one pair in the
    reference's loop order (r1 in kept(I1 = Ij) outer, rp in kept(Ip = Ii) inner): Ei, Ej the
    abs_zero energies of the kept states, o1, o2 the kept x kept blocks of op(Ij, Ii), Z the
    step's Z_ft. Weight op1 op2 ((-sign) e^{-E1/T} + e^{-Ep/T}) / Z at energy E1 - Ep."""
    E = (Ej[:, None] - Ei[None, :]).ravel()
    stat = ((-sign) * np.exp(-Ej[:, None] / T) + np.exp(-Ei[None, :] / T)) / Z
    return E, (o1 * o2 * stat).ravel()


def mats_pair(EGi, Ki, EGj, Kj, o1, o2, rho_i, rho_j, factor, sign, T, wnf, w):
    """Algo_FDMmats::calc (c++/algo_FDM.hpp:167-217) of one subspace pair: the Matsubara
    values factor * sum (weight / (i w_n - E)), E = Ej - Ei, over the D x D (term1), D x K
    (term2) and K x D (term3) state pairs, i the states of Ii (columns of op1, op2), j those
    of Ij (rows); K = the first Ki (Kj) states, D = the rest. For bosonic operators the D x D
    term at n = 0 with |E| <= WEIGHT_TOL (1e-8, c++/numerics.hpp:318) is -weightA / T."""
    ni, nj = len(EGi), len(EGj)
    G = np.zeros(len(w), dtype=complex)
    if ni == 0 or nj == 0:
        return G
    E = EGj[:, None] - EGi[None, :]
    P = o1 * o2
    wA = P * wnf * np.exp(-EGi / T)[None, :]           # a[ij] b[ji] exp(-beta e[i])
    wB = P * (-sign) * wnf * np.exp(-EGj / T)[:, None]  # a[ij] b[ji] sign exp(-beta e[j])

    def add(wt, e, special=None):
        with np.errstate(invalid="ignore", divide="ignore"):  # the special n = 0 entries are replaced below
            t = wt[:, :, None] / (1j * w[None, None, :] - e[:, :, None])
        if special is not None:
            t[:, :, 0] = np.where(np.abs(e) <= 1e-8, special, t[:, :, 0])
        return t.sum(axis=(0, 1))
    if Ki < ni and Kj < nj:  # term1
        a, b, e = wA[Kj:, Ki:], wB[Kj:, Ki:], E[Kj:, Ki:]
        G += add(a + b, e, -a / T if sign == 1 else None)
    if Ki < ni and Kj > 0:  # term2: rho_op2 = prod_fit(rhoFDM(Ij), op2)
        r = rho_j.shape[0]
        rho_op2 = rho_j @ o2[:r, :]
        G += add(wA[:Kj, Ki:] + (-sign) * o1[:Kj, Ki:] * rho_op2[:Kj, Ki:], E[:Kj, Ki:])
    if Ki > 0 and Kj < nj:  # term3: op2_rho = prod_fit(op2, rhoFDM(Ii))
        r = rho_i.shape[0]
        op2_rho = o2[:, :r] @ rho_i
        G += add(o1[Kj:, :Ki] * op2_rho[Kj:, :Ki] + wB[Kj:, :Ki], E[Kj:, :Ki])
    return factor * G


def mats_sum(wt, E, w, special=None):
    """sum over the (j, i) terms of wt / (i w_n - E) for every Matsubara point w_n; `special`
    replaces the n = 0 terms with |E| <= WEIGHT_TOL (1e-8) when given (bosonic operators)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        t = wt[:, :, None] / (1j * w[None, None, :] - E[:, :, None])
    if special is not None:
        t[:, :, 0] = np.where(np.abs(E) <= 1e-8, special, t[:, :, 0])
    return t.sum(axis=(0, 1))


def dmnrg_mats_pair(Em, Ej, o1, o2, rho_p, rho_1, factor, sign, T, w):
    """Algo_DMNRGmats::calc (c++/algo_DMNRG.hpp:76-100) of one pair over kept(Ip) x kept(I1):
    weightA = (sum_ri op2(rj, ri) rho(Ip)(rm, ri)) op1(rj, rm), weightB = (sum_ri op1(ri, rm)
    rho(I1)(rj, ri)) op2(rj, rm), term (weightA - sign weightB) / (i w_n - (Ej - Em)); for a
    bosonic operator at n = 0 and |Ej - Em| <= 1e-8 the term is -weightA / T."""
    if o1.size == 0:
        return np.zeros(len(w), dtype=complex)
    wA = (o2 @ rho_p.T) * o1
    wB = (rho_1 @ o1) * o2
    E = Ej[:, None] - Em[None, :]
    return factor * mats_sum(wA + (-sign) * wB, E, w, -wA / T if sign == 1 else None)


def ft_mats_pair(Ep, E1, o1, o2, Z, factor, sign, T, w):
    """Algo_FTmats::calc (c++/algo_FT.hpp:63-85) of one pair over kept(I1) x kept(Ip):
    op1 op2 ((-sign) e^{-E1/T} + e^{-Ep/T}) / (Z (i w_n - (E1 - Ep))); for a bosonic operator at
    n = 0 and |E1 - Ep| <= 1e-8 the term is -op1 op2 e^{-E1/T} / (Z T)."""
    if o1.size == 0:
        return np.zeros(len(w), dtype=complex)
    P = o1 * o2
    E = E1[:, None] - Ep[None, :]
    wt = P * ((-sign) * np.exp(-E1 / T)[:, None] + np.exp(-Ep / T)[None, :]) / Z
    return factor * mats_sum(wt, E, w, -P * np.exp(-E1 / T)[:, None] / (Z * T) if sign == 1 else None)


def _dm_outputs(kv, steps, Lam, disc, z, Nmax, specs, algos, out, fdm_out, GS, combs, singlet_names, bins_out=None,
                init_spec=None):
    """The DMNRG run (c++/nrg-general.hpp:139-168): the density matrices (calc_rho +
    calc_densitymatrix for DMNRG, c++/dmnrg.hpp:43-133; calc_rhoFDM for FDM,
    c++/dmnrg.hpp:146-217), then per step the spectra of every algorithm
    (BaseSpectrum::calc, c++/algo.hpp:55-67): Algo_DMNRG merged with the N/N+2 window
    (mergeNN2), Algo_FDMgt/ls merged whole (mergeCFS); at the end trim + continuous
    (log-Gaussian broadening). FDM expectation values at step fdmexpvn
    (measure_singlet_fdm, c++/measurements.hpp:31-44)."""
    T = float(kv.get("T", 0.001))
    brs = float(kv.get("bandrescale", 1.0))
    goodE = float(kv.get("goodE", 2.0))
    bins = int(kv.get("bins", 1000))
    NN1 = kv.get("NN1", "false").lower() == "true"
    NN2avg = kv.get("NN2avg", "false").lower() == "true"
    NN2even = kv.get("NN2even", "true").lower() == "true"
    NNtanh = float(kv.get("NNtanh", 0.0))
    discard_trim = float(kv.get("discard_trim", 1e-16))
    reim = kv.get("reim", "false").lower() == "true"
    broaden_on = kv.get("broaden", "true").lower() == "true"
    discard_imm = float(kv.get("discard_immediately", 1e-16))
    emin_p, emax_p = float(kv.get("emin", -1.0)), float(kv.get("emax", -1.0))
    alpha = float(kv.get("alpha", 0.3))
    omega0 = float(kv.get("omega0", -1.0))
    if omega0 < 0.0:
        omega0 = float(kv.get("omega0_ratio", 1.0)) * T
    bmax = float(kv.get("broaden_max", 10.0))
    bmin = float(kv.get("broaden_min", -99.0))
    bratio = float(kv.get("broaden_ratio", 1.05))
    fdmexpvn = int(kv.get("fdmexpvn", 0))
    nmats = int(kv.get("mats", 100))
    last_scale = SCALE(Nmax, Lam, disc, z, brs)
    if bmin <= 0.0:
        bmin = float(kv.get("broaden_min_ratio", 3.0)) * last_scale
    Efac = Lam if (combs == 4 and not NN1) else math.sqrt(Lam)  # Params::getEfactor (c++/params.hpp:650-652)
    nst = len(steps)
    IN = _qs.QS1.IN if combs == 4 else _qs.QS2.IN

    def sweep(rho_last, extra):
        """calc_densitymatrix_iterN / calc_fulldensitymatrix_iterN (c++/dmnrg.hpp:85-102,
        165-197) with cdmI (55-80): rho at step k-1 from rho and `extra(k)` at step k."""
        rhos = {nst - 1: rho_last}
        for k in range(nst - 1, 0, -1):
            _, _, diagN, structN, _, _ = steps[k]
            _, _, diagP, _, _, _ = steps[k - 1]
            terms = [rhos[k]] + ([extra(k)] if extra and k < nst - 1 else [])  # no DD sector at the last step
            prev = {}
            for I, eP in diagP.items():
                dim = eP.nrpost
                M = np.zeros((dim, dim))
                if dim:
                    for i, dl in enumerate(IN):
                        sub = (I[0] - dl[0], I[1] - dl[1])
                        if sub not in diagN:
                            continue
                        for rhoN in terms:
                            if sub not in rhoN:
                                continue
                            nw = rhoN[sub].shape[0]
                            rmax = structN[sub][1][i]
                            if nw == 0 or rmax == 0:
                                continue
                            assert rmax == dim
                            U = np.ascontiguousarray(diagN[sub].U[i][:nw])
                            O.rotate(M, float(sub[1]) / float(I[1]), U, np.ascontiguousarray(rhoN[sub]))
                prev[I] = M
            rhos[k - 1] = prev
        return rhos

    def trace(rho):
        return sum(I[1] * np.trace(m) for I, m in rho.items())

    rhos = fdm = None
    Zft = None
    if "DMNRG" in algos or "DMNRGmats" in algos or any(a.startswith("CFS") for a in algos):  # Params::need_rho
        # init_rho over the kept states of the last step (c++/dmnrg.hpp:43-50)
        _, scale_last, diag_last, _, _, _ = steps[-1]
        scT = scale_last / T
        Z = sum(I[1] * sum(math.exp(-c * scT) for c in e.corr[:e.nrpost]) for I, e in diag_last.items())
        rho = {I: np.diag([math.exp(-c * scT) for c in e.corr[:e.nrpost]]) / Z for I, e in diag_last.items()}
        Zft = Z  # calc_Z at the last step (c++/measurements.hpp:189-191): the same kept-state sum
        rhos = sweep(rho, None)
        for k in range(nst):
            assert abs(trace(rhos[k]) - 1.0) < 1e-10
    if fdm_out is not None or any(a.startswith("FDM") for a in algos):
        wn, wnfactor, ZnDNd, tdrow = _fdm_weights(steps, T, GS, combs)

        def init_rho_fdm(k):
            """init_rho_FDM (c++/dmnrg.hpp:146-162): the D states of step k, all states at the
            last step; the matrix spans all states."""
            _, scale, diagN, _, _, _ = steps[k]
            last = k == nst - 1
            r = {}
            for I, e in diagN.items():
                tot = len(e.values)
                m = np.zeros((tot, tot))
                if ZnDNd[k] != 0.0:
                    for i in range(0 if last else e.nrpost, tot):
                        m[i, i] = math.exp(-((e.values[i] - e.shift) * scale) / T) * wn[k] / ZnDNd[k]
                r[I] = m
            if wn[k] != 0.0:
                tr = trace(r)
                if abs((tr - wn[k]) / wn[k]) > 1e-8:
                    assert wn[k] < 1e-12
            return r
        fdm = sweep(init_rho_fdm(nst - 1), init_rho_fdm)
        for k in range(nst - 1):
            expected = sum(wn[k + 1:])
            assert abs((trace(fdm[k]) - expected) / expected) < 1e-10, (k, trace(fdm[k]), expected)
        if fdm_out is not None:
            fdm_out["tdfdm"] = (["T", "E_fdm", "C_fdm", "F_fdm", "S_fdm"], tdrow)
            if kv.get("fdmexpv", "false").lower() == "true" and fdmexpvn < nst:
                _, _, diagN, _, opsN, _ = steps[fdmexpvn]
                row = [T]
                for name in singlet_names:
                    v = 0.0
                    for I, r in fdm[fdmexpvn].items():  # trace_contract over the kept range
                        k_ = diagN[I].nrpost
                        n = opsN["s"][name][(I, I)]
                        v += I[1] * float(np.sum(r[:k_, :k_] * n[:k_, :k_].T))
                    row.append(v)
                fdm_out["customfdm"] = (["T"] + list(singlet_names), row)
    if out is None or not algos:
        return
    emax = emax_p if emax_p > 0 else SCALE(0, Lam, disc, z, brs) * 100.0
    emin = emin_p if emin_p > 0 else last_scale / 100.0
    lmin, lmax = math.floor(math.log10(emin)), math.ceil(math.log10(emax))
    # gf_type and factor of each kind (c++/oprecalc.hpp:160-195; gf_sign, c++/traits.hpp)
    kinds = {"s": (1, _qs.correlator_factor), "d": (-1, _specdens_factor), "t": (1, _qs.dynamicsusceptibility_factor)}
    mesh = []
    E = bmax
    while E > bmin:
        mesh.append(E)
        E /= bratio
    for prefix, kind, name1, name2 in specs:
        sign, ff = kinds[kind]
        full = {a: O.ChainBinning(lmin, lmax, bins, discard_imm) for a in algos if not a.endswith("mats")}
        # GFMatsubara of the Matsubara algorithms (c++/spectrum.hpp:212-227): mats points
        # w_n = ww(n, gt, T), every step's sums merged whole
        wmats = T * math.pi * (2 * np.arange(nmats) + (0 if sign == 1 else 1))
        gm = {a: np.zeros(nmats, dtype=complex) for a in algos if a.endswith("mats")}
        if "FTmats" in algos and init_spec is not None:  # the initial cluster (docalc0), all states kept
            scale0, vals0, opsets0 = init_spec
            o1s, o2s = opsets0[kind].get(name1, {}), opsets0[kind].get(name2, {})
            Z0 = sum(I[1] * float(np.sum(np.exp(-v * scale0 / T))) for I, v in vals0.items())
            for Ii in vals0:
                for Ij in vals0:
                    key = (Ij, Ii)
                    if key in o1s and key in o2s and o1s[key].size:
                        gm["FTmats"] += ft_mats_pair(vals0[Ii] * scale0, vals0[Ij] * scale0, o1s[key], o2s[key], Z0,
                                                     ff(Ii, Ij), sign, T, wmats)
        for k, (N, scale, diagN, _, opsets, Tshift) in enumerate(steps):
            op1, op2 = opsets[kind][name1], opsets[kind][name2]
            last = k == nst - 1
            pairs = []
            for Ii, ei in diagN.items():
                for Ij, ej in diagN.items():
                    if (Ij, Ii) in op1 and (Ij, Ii) in op2 and op1[(Ij, Ii)].size:
                        pairs.append((Ii, ei, Ij, ej))
            if "DMNRG" in algos and (NN1 or NN2avg or (N % 2 == 0 if NN2even else N % 2 == 1)):
                cb = O.ChainBinning(lmin, lmax, bins, discard_imm)
                Emin_w, Emax_w = scale * goodE, scale * goodE * Efac * Efac
                for Ii, ei, Ij, ej in pairs:
                    ki, kj = ei.nrpost, ej.nrpost
                    Em = (ei.values[:ki] - ei.shift) * scale
                    Ej = (ej.values[:kj] - ej.shift) * scale
                    cb.dmnrg_pair(Em, Ej, op1[(Ij, Ii)][:kj, :ki], op2[(Ij, Ii)][:kj, :ki], rhos[k][Ii], rhos[k][Ij],
                                  ff(Ii, Ij), sign, Emin_w, Emax_w)
                Ex = scale * goodE * Efac
                flags = (1 if N == Nmax - 1 else 0) | (2 if N == 0 else 0)
                fs = full["DMNRG"]
                for fr, fi, cr, ci in ((fs.pos_re, fs.pos_im, cb.pos_re, cb.pos_im),
                                       (fs.neg_re, fs.neg_im, cb.neg_re, cb.neg_im)):
                    O.lib().oracle_merge_nn2half(O._ptr(fr), O._ptr(fi), O._ptr(cr), O._ptr(ci), O._ptr(fs.energies),
                                                 fs.nbins, Emin_w, Ex, Emax_w, flags, NNtanh, 1 if NN2avg else 0)
            if "FT" in algos and (NN1 or NN2avg or (N % 2 == 0 if NN2even else N % 2 == 1)):
                # Algo_FT with stats.Zft of this step (calc_Z, c++/measurements.hpp:189-191), merged
                # with the N/N+2 window as DMNRG (mergeNN2)
                scT = scale / T
                Zk = sum(I[1] * sum(math.exp(-c * scT) for c in e.corr[:e.nrpost]) for I, e in diagN.items())
                cb = O.ChainBinning(lmin, lmax, bins, discard_imm)
                for Ii, ei, Ij, ej in pairs:
                    ki, kj = ei.nrpost, ej.nrpost
                    if not (ki and kj):
                        continue
                    E, wt = ft_terms((ei.values[:ki] - ei.shift) * scale, (ej.values[:kj] - ej.shift) * scale,
                                     op1[(Ij, Ii)][:kj, :ki], op2[(Ij, Ii)][:kj, :ki], sign, T, Zk)
                    cb.add(E, wt, ff(Ii, Ij))
                Emin_w, Emax_w = scale * goodE, scale * goodE * Efac * Efac
                Ex = scale * goodE * Efac
                flags = (1 if N == Nmax - 1 else 0) | (2 if N == 0 else 0)
                fs = full["FT"]
                for fr, fi, cr, ci in ((fs.pos_re, fs.pos_im, cb.pos_re, cb.pos_im),
                                       (fs.neg_re, fs.neg_im, cb.neg_re, cb.neg_im)):
                    O.lib().oracle_merge_nn2half(O._ptr(fr), O._ptr(fi), O._ptr(cr), O._ptr(ci), O._ptr(fs.energies),
                                                 fs.nbins, Emin_w, Ex, Emax_w, flags, NNtanh, 1 if NN2avg else 0)
            cfs_algos = [a for a in algos if a.startswith("CFS")]
            if cfs_algos:
                # Algo_CFSgt / Algo_CFSls::calc (c++/algo_CFS.hpp:28-53, 80-105) with Ip = Ii,
                # I1 = Ij; op(r1, rp) has r1 in Ij, rp in Ii; abs_zero energies of all states
                cbs = {w: O.ChainBinning(lmin, lmax, bins, discard_imm) for w in ("gt", "ls")}
                for Ii, ei, Ij, ej in pairs:
                    ki, kj = ei.nrpost, ej.nrpost
                    Ei = (ei.values - ei.shift) * scale
                    Ej = (ej.values - ej.shift) * scale
                    terms = cfs_terms(last, Ei, ki, Ej, kj, op1[(Ij, Ii)], op2[(Ij, Ii)],
                                      None if last else rhos[k][Ii], None if last else rhos[k][Ij], sign, T, Zft)
                    for w, (E, wt) in terms.items():
                        if E.size:
                            cbs[w].add(E, wt, ff(Ii, Ij))
                for a in cfs_algos:  # mergeCFS
                    for w in {"CFS": ("gt", "ls"), "CFSgt": ("gt",), "CFSls": ("ls",)}[a]:
                        for arr in ("pos_re", "pos_im", "neg_re", "neg_im"):
                            getattr(full[a], arr)[:] += getattr(cbs[w], arr)
            if "DMNRGmats" in algos:
                for Ii, ei, Ij, ej in pairs:
                    ki, kj = ei.nrpost, ej.nrpost
                    gm["DMNRGmats"] += dmnrg_mats_pair((ei.values[:ki] - ei.shift) * scale,
                                                       (ej.values[:kj] - ej.shift) * scale, op1[(Ij, Ii)][:kj, :ki],
                                                       op2[(Ij, Ii)][:kj, :ki], rhos[k][Ii], rhos[k][Ij], ff(Ii, Ij),
                                                       sign, T, wmats)
            if "FTmats" in algos:
                scT = scale / T
                Zk = sum(I[1] * sum(math.exp(-c * scT) for c in e.corr[:e.nrpost]) for I, e in diagN.items())
                for Ii, ei, Ij, ej in pairs:
                    ki, kj = ei.nrpost, ej.nrpost
                    gm["FTmats"] += ft_mats_pair((ei.values[:ki] - ei.shift) * scale, (ej.values[:kj] - ej.shift) * scale,
                                                 op1[(Ij, Ii)][:kj, :ki], op2[(Ij, Ii)][:kj, :ki], Zk, ff(Ii, Ij), sign,
                                                 T, wmats)
            if "FDMmats" in algos:
                gmats = gm["FDMmats"]
                for Ii, ei, Ij, ej in pairs:
                    Ki = 0 if last else ei.nrpost
                    Kj = 0 if last else ej.nrpost
                    EGi = ((ei.values - ei.shift) * scale + Tshift) - GS
                    EGj = ((ej.values - ej.shift) * scale + Tshift) - GS
                    gmats += mats_pair(EGi, Ki, EGj, Kj, op1[(Ij, Ii)], op2[(Ij, Ii)], fdm[k][Ii], fdm[k][Ij],
                                       ff(Ii, Ij), sign, T, wnfactor[k], wmats)
            fdm_algos = [a for a in algos if a.startswith("FDM") and a != "FDMmats"]
            if fdm_algos:
                cbs = {w: O.ChainBinning(lmin, lmax, bins, discard_imm) for w in ("gt", "ls")}
                for Ii, ei, Ij, ej in pairs:
                    Ki = 0 if last else ei.nrpost   # Eigen::boundary, c++/eigen.hpp:219
                    Kj = 0 if last else ej.nrpost
                    EGi = ((ei.values - ei.shift) * scale + Tshift) - GS
                    EGj = ((ej.values - ej.shift) * scale + Tshift) - GS
                    for w, rho in (("gt", fdm[k][Ii]), ("ls", fdm[k][Ij])):
                        cbs[w].fdm_pair(w, EGi, Ki, EGj, Kj, op1[(Ij, Ii)], op2[(Ij, Ii)], rho, ff(Ii, Ij), sign, T,
                                        wnfactor[k])
                for a in fdm_algos:  # mergeCFS: Bins::merge (c++/bins.hpp:153-162)
                    parts = {"FDM": ("gt", "ls"), "FDMgt": ("gt",), "FDMls": ("ls",)}[a]
                    for w in parts:
                        for arr in ("pos_re", "pos_im", "neg_re", "neg_im"):
                            getattr(full[a], arr)[:] += getattr(cbs[w], arr)
        for a, g_all in gm.items():  # Matsubara::save with outputxy(..., imagpart=true) (c++/io.hpp:33-38)
            out[f"{prefix}_{a}_dens_{name1}-{name2}"] = np.array(
                [(wn, g.real, g.imag if abs(g.imag) > abs(g.real) * 1e-10 else 0.0) for wn, g in zip(wmats, g_all)])
        for a in algos:
            if a.endswith("mats"):
                continue
            fs = full[a]

            def trim(w):
                e = fs.energies
                keep = [(e[i], w[i]) for i in range(len(e) - 1) if abs(w[i]) >= discard_trim * (e[i + 1] - e[i])]
                keep.append((e[-1], w[-1]))
                return keep
            pos, neg = trim(fs.pos_re), trim(fs.neg_re)
            if bins_out is not None:  # savebins: Bins::trim keeps |w| (complex modulus) >= discard_trim * width
                rows = []
                for sgn, wr, wi in ((1.0, fs.pos_re, fs.pos_im), (-1.0, fs.neg_re, fs.neg_im)):
                    e = fs.energies
                    for i in range(len(e)):
                        if i == len(e) - 1 or abs(complex(wr[i], wi[i])) >= discard_trim * (e[i + 1] - e[i]):
                            rows.append((sgn * e[i], wr[i], wi[i]) if reim else (sgn * e[i], wr[i]))
                bins_out[f"{prefix}_{a}_dens_{name1}-{name2}"] = np.array(rows)
            if not broaden_on:  # SpectrumRealFreq::save: continuous() only with broaden=true
                continue
            rows_pos, rows_neg = [], []
            for E in mesh:
                vp = sum(w * _BR_NEW(E, e, alpha, omega0) for e, w in pos) + \
                    sum(w * _BR_NEW(E, -e, alpha, omega0) for e, w in neg)
                vn = sum(w * _BR_NEW(-E, e, alpha, omega0) for e, w in pos) + \
                    sum(w * _BR_NEW(-E, -e, alpha, omega0) for e, w in neg)
                rows_pos.append((E, vp))
                rows_neg.append((-E, vn))
            out[f"{prefix}_{a}_dens_{name1}-{name2}"] = np.array(sorted(rows_neg) + sorted(rows_pos))
