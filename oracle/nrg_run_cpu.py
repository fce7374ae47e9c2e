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
  recalc_doublet (QS)         c++/symmetry/nrg-recalc-QS.hpp:32-117, qs-1ch-doublet{p,m}.dat
  DM-NRG                      init_rho, cdmI, calc_densitymatrix(_iterN) c++/dmnrg.hpp:43-112;
                              Algo_DMNRG c++/algo_DMNRG.hpp:29-52; BaseSpectrum::calc c++/algo.hpp:55-67;
                              mergeNN2half, windowfunction, continuous c++/spectrum.hpp:81-196;
                              Bins c++/bins.hpp:61-185; BR_NEW c++/spectral.hpp:42-70

Only ``tests/`` and the CPU-baseline leg of ``bench.py`` may import this module.
"""
from __future__ import annotations

import math
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


def run(param_text: str, data_text: str, threads: int = 1, spectra: dict = None
        ) -> Tuple[List[str], List[List[float]], List[str], List[List[float]]]:
    """td and custom rows of the run; with dmnrg=true and a `spectra` dict, also the DM-NRG
    spectra of the specs, specd and spect pairs (file stem, e.g. spec_DMNRG_dens_A_d-A_d ->
    array of (E, A(E)) rows as written to that .dat file)."""
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
    flag = lambda k: kv.get(k, "false").lower() == "true"  # noqa: E731
    # Params::keep_all_states_in_last_step (c++/params.hpp:535-539)
    lastall = flag("lastall") or ((flag("fdm") or flag("fdmexpv")) and not flag("lastalloverride"))
    rescaled = kv.get("data_has_rescaled_energies", "true").lower() == "true"
    d = read_data(data_text)
    Nmax = d.nmax
    T = _qs.tables(d.channels)
    _IN, _QN, C = T.IN, T.QN, T.COMBS
    O.blas_threads(1)  # one BLAS thread per block, as diagonalisations_OpenMP runs dsyev

    def scale_of(trueN):
        return SCALE(trueN + 1, Lam, disc, z)

    diag: Dict = {}
    for I, e in sorted(d.subspaces):
        v = e.copy() if rescaled else e / SCALE(0, Lam, disc, z)
        diag[I] = _Eig(v)
    opch = [dict(d.opch[ch][0]) for ch in range(d.channels)]
    ops = {name: {I1: m for (I1, I2), m in mats.items() if I1 == I2}
           for name, (kind, mats) in d.ops.items() if kind in "sg"}
    dm = kv.get("dmnrg", "false").lower() == "true" and spectra is not None

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
            for i in range(C):
                for n in range(dims[i]):
                    h[off[i] + n, off[i] + n] = math.sqrt(Lam) * diag[anc[i]].corr[n]
            for (i, j, ch, fn) in T.OFFDIAG:
                if dims[i - 1] and dims[j - 1]:
                    fs = (fn(I[1]) * d.xi[ch][N]) / scale
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
        # after_diag
        td(N, new)
        for I, e in new.items():
            anc, dims = structure[I]
            off = np.concatenate([[0], np.cumsum(dims)]).astype(int)
            e.U = [np.ascontiguousarray(e.vectors[:, off[i]:off[i + 1]]) for i in range(C)]

        def recalc_ops(nrows):
            out = {}
            for name in sorted(ops):
                cold = ops[name]
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
                            O.product(f, fn(Ip[1]), A, B)
                    nf[ch][(I1, Ip)] = f
            opch = nf
        if strategy == "kept":
            ops = recalc_ops(lambda e: e.nrstored)
            custom(N, new, ops)
        if dm:
            def recalc_tensor(cold, tables, factor):
                """recalc_general (c++/recalc.hpp:82-108) over the pairs Ip = I1 + dq."""
                cn = {}
                for I1, e1 in new.items():
                    for dq, table in tables:
                        Ip = (I1[0] + dq[0], I1[1] + dq[1])
                        if Ip not in new or not (e1.nrstored and new[Ip].nrstored):
                            continue
                        ep = new[Ip]
                        m = np.zeros((e1.nrstored, ep.nrstored))
                        anc1, dims1 = structure[I1]
                        ancp, dimsp = structure[Ip]
                        for i1, ip, fn in table:
                            IN1, INp = anc1[i1 - 1], ancp[ip - 1]
                            if IN1[1] <= 0 or INp[1] <= 0 or (IN1, INp) not in cold:
                                continue
                            if dims1[i1 - 1] == 0 or dimsp[ip - 1] == 0:
                                continue
                            A = np.ascontiguousarray(e1.U[i1 - 1][:e1.nrstored])
                            B = np.ascontiguousarray(ep.U[ip - 1][:ep.nrstored])
                            Oa = np.ascontiguousarray(cold[(IN1, INp)][:dims1[i1 - 1], :dimsp[ip - 1]])
                            O.transform(m, factor(fn, I1[1]), A, Oa, B)
                        cn[(I1, Ip)] = m
                return cn
            # recalc_doublet (nrg-recalc-QS.hpp:32-117), recalc_triplet (495-640)
            dops = {name: recalc_tensor(cold, (((-1, 1), _DOUBLETP), ((-1, -1), _DOUBLETM)), lambda fn, ss: fn(ss))
                    for name, cold in dops.items()}
            tops = {name: recalc_tensor(cold, T.TRIPLET, _qs.triplet_factor) for name, cold in tops.items()}
            sops = {name: {(I, I): m for I, m in ops[name].items()} for name in {x for sp in specs if sp[1] == "s"
                                                                                 for x in sp[2:]}}
            steps.append((N, scale, new, structure, {"s": sops, "d": dops, "t": tops}))
        diag = new
    if dm and steps:
        _dmnrg_spectra(kv, steps, Lam, disc, z, Nmax, specs, spectra)
    td_fields = ["T", "<Sz^2>", "<Q>", "<Q^2>", "<E>", "<E^2>", "C", "F", "S"]
    return td_fields, td_rows, ["T"] + sorted(ops), custom_rows


def _dmnrg_spectra(kv, steps, Lam, disc, z, Nmax, specs, out):
    """calc_rho + calc_densitymatrix, then the DMNRG run's spectral part: per step
    Algo_DMNRG::calc over all subspace pairs, mergeNN2 into the full spectrum, and at the end
    trim + continuous (log-Gaussian broadening)."""
    T = float(kv.get("T", 0.001))
    goodE = float(kv.get("goodE", 2.0))
    bins = int(kv.get("bins", 1000))
    NN1 = kv.get("NN1", "false").lower() == "true"
    NN2avg = kv.get("NN2avg", "false").lower() == "true"
    NN2even = kv.get("NN2even", "true").lower() == "true"
    NNtanh = float(kv.get("NNtanh", 0.0))
    discard_trim = float(kv.get("discard_trim", 1e-16))
    discard_imm = float(kv.get("discard_immediately", 1e-16))
    emin_p, emax_p = float(kv.get("emin", -1.0)), float(kv.get("emax", -1.0))
    alpha = float(kv.get("alpha", 0.3))
    omega0 = float(kv.get("omega0", -1.0))
    if omega0 < 0.0:
        omega0 = float(kv.get("omega0_ratio", 1.0)) * T
    bmax = float(kv.get("broaden_max", 10.0))
    bmin = float(kv.get("broaden_min", -99.0))
    bratio = float(kv.get("broaden_ratio", 1.05))
    last_scale = SCALE(Nmax, Lam, disc, z)
    if bmin <= 0.0:
        bmin = float(kv.get("broaden_min_ratio", 3.0)) * last_scale
    Efac = Lam  # one channel, no N/N+1 patching
    if NN1:
        Efac = math.sqrt(Lam)
    # density matrix at the last step over the kept states (init_rho)
    N_last, scale_last, diag_last, _, _ = steps[-1]
    scT = scale_last / T
    Z = sum(I[1] * sum(math.exp(-c * scT) for c in e.corr[:e.nrstored]) for I, e in diag_last.items())
    rho = {I: np.diag([math.exp(-c * scT) for c in e.corr[:e.nrstored]]) / Z for I, e in diag_last.items()}
    rhos = {N_last: rho}
    for k in range(len(steps) - 1, 0, -1):
        N, _, diagN, structN, _ = steps[k]
        _, _, diagP, _, _ = steps[k - 1]
        rhoN = rhos[N]
        prev = {}
        for I, eP in diagP.items():
            dim = eP.nrstored
            M = np.zeros((dim, dim))
            if dim:
                for i, dl in enumerate(_qs.QS1.IN):
                    sub = (I[0] - dl[0], I[1] - dl[1])
                    if sub not in rhoN or sub not in diagN:
                        continue
                    nw = rhoN[sub].shape[0]
                    rmax = structN[sub][1][i]
                    if nw == 0 or rmax == 0:
                        continue
                    assert rmax == dim
                    U = np.ascontiguousarray(diagN[sub].U[i][:nw])
                    O.rotate(M, float(sub[1]) / float(I[1]), U, np.ascontiguousarray(rhoN[sub]))
            prev[I] = M
        tr = sum(I[1] * np.trace(m) for I, m in prev.items())
        assert abs(tr - 1.0) < 1e-10, tr
        rhos[N - 1] = prev
    emax = emax_p if emax_p > 0 else SCALE(0, Lam, disc, z) * 100.0
    emin = emin_p if emin_p > 0 else last_scale / 100.0
    lmin, lmax = math.floor(math.log10(emin)), math.ceil(math.log10(emax))
    # gf_type and factor of each kind (c++/oprecalc.hpp:160-195; gf_sign, c++/traits.hpp)
    kinds = {"s": (1, _qs.correlator_factor), "d": (-1, _specdens_factor), "t": (1, _qs.dynamicsusceptibility_factor)}
    for prefix, kind, name1, name2 in specs:
        sign, ff = kinds[kind]
        full = O.ChainBinning(lmin, lmax, bins, discard_imm)
        for N, scale, diagN, _, dopsN in steps:
            merge = NN1 or NN2avg or (N % 2 == 0 if NN2even else N % 2 == 1)
            if not merge:
                continue
            cb = O.ChainBinning(lmin, lmax, bins, discard_imm)
            rhoN = rhos[N]
            Emin_w, Emax_w = scale * goodE, scale * goodE * Efac * Efac
            op1, op2 = dopsN[kind][name1], dopsN[kind][name2]
            for Ii, ei in diagN.items():
                for Ij, ej in diagN.items():
                    if (Ij, Ii) not in op1 or (Ij, Ii) not in op2:
                        continue
                    if ei.nrstored == 0 or ej.nrstored == 0:
                        continue
                    Em = (ei.values[:ei.nrstored] - ei.shift) * scale
                    Ej = (ej.values[:ej.nrstored] - ej.shift) * scale
                    cb.dmnrg_pair(Em, Ej, op1[(Ij, Ii)], op2[(Ij, Ii)], rhoN[Ii], rhoN[Ij], ff(Ii, Ij), sign,
                                  Emin_w, Emax_w)
            Ex = scale * goodE * Efac
            flags = (1 if N == Nmax - 1 else 0) | (2 if N == 0 else 0)
            for fr, fi, cr, ci in ((full.pos_re, full.pos_im, cb.pos_re, cb.pos_im),
                                   (full.neg_re, full.neg_im, cb.neg_re, cb.neg_im)):
                O.lib().oracle_merge_nn2half(O._ptr(fr), O._ptr(fi), O._ptr(cr), O._ptr(ci), O._ptr(full.energies),
                                             full.nbins, Emin_w, Ex, Emax_w, flags, NNtanh, 1 if NN2avg else 0)

        def trim(w):
            e = full.energies
            keep = [(e[i], w[i]) for i in range(len(e) - 1) if abs(w[i]) >= discard_trim * (e[i + 1] - e[i])]
            keep.append((e[-1], w[-1]))
            return keep
        pos, neg = trim(full.pos_re), trim(full.neg_re)
        mesh = []
        E = bmax
        while E > bmin:
            mesh.append(E)
            E /= bratio
        rows_pos, rows_neg = [], []
        for E in mesh:
            vp = sum(w * _BR_NEW(E, e, alpha, omega0) for e, w in pos) + sum(w * _BR_NEW(E, -e, alpha, omega0) for e, w in neg)
            vn = sum(w * _BR_NEW(-E, e, alpha, omega0) for e, w in pos) + sum(w * _BR_NEW(-E, -e, alpha, omega0) for e, w in neg)
            rows_pos.append((E, vp))
            rows_neg.append((-E, vn))
        out[f"{prefix}_DMNRG_dens_{name1}-{name2}"] = np.array(sorted(rows_neg) + sorted(rows_pos))
