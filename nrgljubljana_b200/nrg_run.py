"""NRG iteration for symmetry QS (one channel) on the B200 step core.

Host mirror of the reference's run loop -- docalc0 (c++/core.hpp:251-260), nrg_loop
(c++/core.hpp:286-293), iterate / do_diag / after_diag (c++/core.hpp:122-248) -- in which
every O(n^2) and O(n^3) step runs on the device through the C-ABI of libnrg_b200:

  hamiltonian() + make_matrix()       nrg_hamiltonian_batch   (all blocks, one launch)
  diagonalisations()                  nrg_diag_batch          (all blocks, one call)
  recalc_irreducible / recalc_f       nrg_gemm3_batch         (product terms)
  recalculate_operators / singlets    nrg_gemm3_batch         (transform terms)

Matrices (block Hamiltonians, eigenvectors, <||f||> and operator matrices) stay in device
memory for the whole run. The host keeps what is O(states): the eigenvalues (one copy per
step), the ground-state subtraction, the splitting correction (c++/splitting.hpp:34-73),
the truncation (c++/truncation.hpp:14-69) and the thermodynamics
(c++/measurements.hpp:166-186, 18-30), computed in the reference's order.

Scope: symtype=QS with one channel, no substeps, Ninit=0, energies rescaled (not
``absolute``), full diagonalisation (``diagratio`` = 1), strategy ``kept`` or ``all``,
singlet operators (``s`` and ``g`` blocks). Anything else is rejected.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import qs
from ._lib import HPiece, NRG_HP_BLOCK, NRG_HP_DIAG, NRGError
from .api import Context, context, diag_batch_device, gemm3, gemm3_batch, _stream_ptr
from .inputs import DataFile, SCALE, parse_param, read_data

Invar = Tuple[int, int]

# Parameters that do not change td/custom of a run without spectral functions.
_IGNORED = {
    "symtype", "model", "U", "Gamma", "delta", "band", "T", "Tmin", "checksumrules", "logall", "log",
    "dumpannotated", "dumpscaled", "dumpabs", "dumpgroups", "dumpenergies", "ops", "diag", "diagth",
    "Nmax", "prec_td", "prec_custom", "width_td", "width_custom", "specs", "specd", "spect",
}


@dataclass
class RunParams:
    """The parameters of c++/params.hpp that shape a QS run's thermodynamics."""
    Lambda: float = 2.0
    z: float = 1.0
    discretization: str = "Z"
    bandrescale: float = 1.0
    keep: int = 100
    keepenergy: float = -1.0
    keepmin: int = 0
    safeguard: float = 1e-5
    safeguardmax: int = 200
    fixeps: float = 1e-15
    betabar: float = 1.0
    strategy: str = "kept"
    calc0: bool = True
    lastall: bool = False
    data_has_rescaled_energies: bool = True

    @classmethod
    def from_param(cls, kv: Dict[str, str]) -> "RunParams":
        p = cls()
        conv = {f: type(getattr(p, f)) for f in p.__dataclass_fields__}
        for k, v in kv.items():
            if k in conv:
                t = conv[k]
                setattr(p, k, (v.lower() == "true") if t is bool else t(v))
            elif k == "diagratio":
                if float(v) != 1.0:
                    raise ValueError("partial diagonalisation (diagratio < 1) is not supported")
            elif k == "Ninit":
                if int(v) != 0:
                    raise ValueError("Ninit != 0 is not supported")
            elif k in ("absolute", "substeps") and v.lower() == "true":
                raise ValueError(f"{k}=true is not supported")
            elif k not in _IGNORED and k not in ("absolute", "substeps"):
                raise ValueError(f"parameter {k} is not supported by the QS run driver")
        if p.strategy not in ("kept", "all"):
            raise ValueError(f"strategy={p.strategy}")
        return p


@dataclass
class Result:
    td_fields: List[str]
    td: List[List[float]]
    custom_fields: List[str]
    custom: List[List[float]]
    blocks_per_step: List[int] = field(default_factory=list)
    max_dim_per_step: List[int] = field(default_factory=list)


# ------------------------------------------------------------------ host bookkeeping
def cluster_mapping(energies: np.ndarray, eps: float) -> Dict[float, float]:
    """Clusters(diag, epsilon) of c++/splitting.hpp:48-72 over the sorted energies: maps the
    members of a split cluster to its lowest value. The loop, as in the reference, counts
    the first element twice and never closes the last cluster."""
    mapping: Dict[float, float] = {}
    e = energies
    e0, i0, size = e[0], 0, 1
    for i in range(len(e)):
        if e[i] - e0 < eps:
            size += 1
        else:
            if size > 1:
                seg = e[i0:i]
                if np.any(seg != seg[0]):
                    for j in range(i0 + 1, i):
                        if e[j] != e[i0]:
                            mapping.setdefault(float(e[j]), float(e[i0]))
            e0, i0, size = e[i], i, 1
    return mapping


def highest_retained_energy(energies: np.ndarray, p: RunParams) -> float:
    """c++/truncation.hpp:14-34 (energies sorted, corrected, unscale = 1)."""
    total = len(energies)
    if energies[0] != 0.0:
        raise AssertionError("energies.front() == 0.0")
    if p.keepenergy <= 0.0:
        nrkeep = p.keep
    else:
        nrkeep = 1 + int(np.count_nonzero(energies <= p.keepenergy))
        nrkeep = min(max(nrkeep, p.keepmin), p.keep)
    if p.safeguard > 0.0:
        extra = 0
        while nrkeep < total and (energies[nrkeep] - energies[nrkeep - 1]) <= p.safeguard and extra < p.safeguardmax:
            nrkeep += 1
            extra += 1
    nrkeep = min(max(nrkeep, 1), total)
    return float(energies[nrkeep - 1])


@dataclass
class Sub:
    """One subspace of a step: host eigenvalues and the device eigenvector rows."""
    I: Invar
    values: np.ndarray                 # computed eigenvalues (relative), ascending
    shift: float = 0.0
    corr: Optional[np.ndarray] = None  # corrected values (splitting fix), all computed
    nstored: int = 0                   # states kept after truncate_perform (all before)
    nkept: int = 0
    dims: List[int] = field(default_factory=list)  # ancestor block widths
    offs: List[int] = field(default_factory=list)
    vec: Optional[torch.Tensor] = None  # n x n (device), row r = eigenvector r

    def block(self, i: int, rows: int) -> torch.Tensor:
        """U(i) restricted to the first `rows` states (split_in_blocks, c++/recalc.hpp:18-30)."""
        return self.vec[:rows, self.offs[i]:self.offs[i] + self.dims[i]]


class QSRun:
    """One NRG run (QS, one channel) on one device."""

    def __init__(self, params: RunParams, data: DataFile, device: int = 0, ctx: Optional[Context] = None):
        if data.symtype != "QS" or data.channels != 1:
            raise ValueError("the driver covers symtype QS with one channel")
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the QS run driver has no CPU fallback")
        self.p = params
        self.d = data
        self.dev = torch.device("cuda", device)
        self.ctx = ctx or context(device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.nmax = data.nmax
        self.sqrt_lambda = math.sqrt(params.Lambda)  # nrg_step_scale_factor (c++/params.hpp:639-641)

    # ---- scales (c++/step.hpp:30-39)
    def scale(self, trueN: int) -> float:
        return SCALE(trueN + 1, self.p.Lambda, self.p.discretization, self.p.z, self.p.bandrescale)

    def _to_dev(self, a: np.ndarray) -> torch.Tensor:
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.dev, non_blocking=False)

    # ---- measurements
    def _td(self, trueN: int, diag: Dict[Invar, Sub]) -> List[float]:
        f = self.p.betabar  # TD_factor (unscale = 1)
        Z = E = E2 = 0.0
        Zs = []
        for I, s in diag.items():
            x = s.values - s.shift
            ex = np.exp(-f * x)
            m = qs.mult(I)
            Z += m * float(np.sum(ex))
            E += m * float(np.sum((f * x) * ex))
            E2 += m * float(np.sum((f * x) ** 2 * ex))
            Zs.append(m * float(np.sum(np.exp(-f * s.corr[:s.nstored]))))
        T = self.scale(trueN) / self.p.betabar
        extra = qs.td_extra(Zs, list(diag.keys()), Z)
        return [T] + extra + [E / Z, E2 / Z, E2 / Z - (E / Z) ** 2, -math.log(Z), E / Z + math.log(Z)]

    def _custom(self, trueN: int, diag: Dict[Invar, Sub], ops: Dict[str, Dict[Invar, torch.Tensor]]) -> List[float]:
        f = self.p.betabar
        Z = 0.0
        for I, s in diag.items():
            Z += qs.mult(I) * float(np.sum(np.exp(-f * s.corr[:s.nstored])))
        row = [self.scale(trueN) / self.p.betabar]
        names = sorted(ops)
        # one device->host copy of every needed diagonal
        diags = []
        for name in names:
            for I, s in diag.items():
                diags.append(torch.diagonal(ops[name][I])[:s.nstored])
        host = torch.cat(diags).cpu().numpy() if diags else np.zeros(0)
        k = 0
        for name in names:
            tr = 0.0
            for I, s in diag.items():
                d = host[k:k + s.nstored]
                k += s.nstored
                tr += qs.mult(I) * float(np.sum(np.exp(-f * s.corr[:s.nstored]) * d))
            row.append(tr / Z)
        return row

    # ---- the run
    def run(self) -> Result:
        p, d = self.p, self.d
        scale0 = SCALE(0, p.Lambda, p.discretization, p.z, p.bandrescale)  # SCALE(Ninit)
        diag: Dict[Invar, Sub] = {}
        for I, e in sorted(d.subspaces):
            v = e.copy() if p.data_has_rescaled_energies else e / scale0
            s = Sub(I, v, 0.0, v.copy(), len(v), len(v))
            diag[I] = s
        opch = {k: self._to_dev(m) for k, m in d.opch[0][0].items()}
        ops: Dict[str, Dict[Invar, torch.Tensor]] = {}
        for name, (kind, mats) in d.ops.items():
            if kind in "sg":
                ops[name] = {I1: self._to_dev(m) for (I1, I2), m in mats.items() if I1 == I2}
        res = Result(["T"] + list(qs.TD_FIELDS) + ["<E>", "<E^2>", "C", "F", "S"], [], ["T"] + sorted(ops), [])
        if p.calc0:
            res.td.append(self._td(-1, diag))
            res.custom.append(self._custom(-1, diag, ops))
        # diag0 has identity eigenvectors: its <||f||> and operators are used as read.
        for N in range(0, self.nmax):
            diag, opch, ops = self._step(N, diag, opch, ops, res)
        return res

    def _step(self, N: int, prev: Dict[Invar, Sub], opch, ops, res: Result):
        p, d = self.p, self.d
        last = N == self.nmax - 1
        scale = self.scale(N)
        # subspace structure (c++/core.hpp:42-58, 62-70; c++/subspaces.hpp:114-121)
        new = set()
        for I in prev:
            for J in qs.new_subspaces(I):
                if qs.allowed(J):
                    new.add(J)
        tasks: List[Tuple[Invar, List[int], List[Invar]]] = []
        for I in sorted(new):
            anc = qs.ancestors(I)
            dims = [(prev[a].nstored if a in prev else 0) if qs.triangle(I, a, qs.QN[i]) else 0
                    for i, a in enumerate(anc)]
            if sum(dims):
                tasks.append((I, dims, anc))
        nb = len(tasks)
        ns = [sum(t[1]) for t in tasks]
        res.blocks_per_step.append(nb)
        res.max_dim_per_step.append(max(ns))
        moff = np.zeros(nb + 1, dtype=np.int64)
        moff[1:] = np.cumsum(np.array(ns, dtype=np.int64) ** 2)
        voff = np.zeros(nb + 1, dtype=np.int64)
        voff[1:] = np.cumsum(ns)
        Hbuf = torch.empty(int(moff[-1]), dtype=torch.float64, device=self.dev)
        Vbuf = torch.empty(int(moff[-1]), dtype=torch.float64, device=self.dev)
        Ebuf = torch.empty(int(voff[-1]), dtype=torch.float64, device=self.dev)
        H = [Hbuf[moff[b]:moff[b + 1]].view(ns[b], ns[b]) for b in range(nb)]
        V = [Vbuf[moff[b]:moff[b + 1]].view(ns[b], ns[b]) for b in range(nb)]
        E = [Ebuf[voff[b]:voff[b + 1]] for b in range(nb)]

        # corrected ancestor energies on the device (one copy)
        pkeys = [I for I in prev if prev[I].nstored > 0]
        poff = {}
        flat = []
        o = 0
        for I in pkeys:
            poff[I] = o
            flat.append(prev[I].corr[:prev[I].nstored])
            o += prev[I].nstored
        pcorr = self._to_dev(np.concatenate(flat)) if flat else None

        # Hamiltonian pieces: hamiltonian() + SymmetryQS::make_matrix
        pieces: List[HPiece] = []
        xi, zeta = d.xi[0], d.zeta[0]
        for b, (I, dims, anc) in enumerate(tasks):
            offs = np.concatenate([[0], np.cumsum(dims)]).astype(int)
            for i in range(qs.COMBS):
                if dims[i]:
                    src = pcorr.data_ptr() + 8 * poff[anc[i]]
                    pieces.append(HPiece(b, NRG_HP_DIAG, int(offs[i]), int(offs[i]), dims[i], dims[i], 0, 0, 0,
                                         src, self.sqrt_lambda, 0.0))
            ss = I[1]
            for (i, j, ch, fn) in qs.OFFDIAG:
                if not (dims[i - 1] and dims[j - 1]):
                    continue
                factor = fn(ss) * xi[N]
                key = (anc[i - 1], anc[j - 1])
                if key not in opch:
                    raise RuntimeError(f"offdiag_function(): matrix not found {i} {j} {ch} 0")
                mat = opch[key]
                if tuple(mat.shape) != (dims[i - 1], dims[j - 1]):
                    raise AssertionError("qq.rmax(i-1) == size1(mat) && qq.rmax(j-1) == size2(mat)")
                fs = factor / scale
                if i > j:
                    pieces.append(HPiece(b, NRG_HP_BLOCK, int(offs[j - 1]), int(offs[i - 1]), dims[j - 1],
                                         dims[i - 1], 1, 0, mat.stride(0), mat.data_ptr(), fs, 0.0))
                else:
                    pieces.append(HPiece(b, NRG_HP_BLOCK, int(offs[i - 1]), int(offs[j - 1]), dims[i - 1],
                                         dims[j - 1], 0, 0, mat.stride(0), mat.data_ptr(), fs, 0.0))
            for (i, ch, number) in qs.DIAG:
                if dims[i - 1]:
                    shift = zeta[N + 1] * (number - 1.0 * qs.AVGOCCUP) / scale
                    pieces.append(HPiece(b, NRG_HP_DIAG, int(offs[i - 1]), int(offs[i - 1]), dims[i - 1],
                                         dims[i - 1], 0, 0, 0, None, 0.0, shift))
        self._assemble(ns, H, pieces)

        info = diag_batch_device(H, E, V, self.ctx, self.stream)
        if np.any(info != 0):
            b = int(np.nonzero(info)[0][0])
            raise RuntimeError(f"dsyev failed. INFO={int(info[b])} (subspace {tasks[b][0]})")
        evals = Ebuf.cpu().numpy()

        diag: Dict[Invar, Sub] = {}
        for b, (I, dims, anc) in enumerate(tasks):
            offs = [int(x) for x in np.concatenate([[0], np.cumsum(dims)])[:-1]]
            diag[I] = Sub(I, evals[voff[b]:voff[b + 1]].copy(), dims=list(dims), offs=offs, vec=V[b],
                          nstored=ns[b])
        # do_diag: Egs subtraction, splitting correction, truncation (c++/core.hpp:141-143)
        Egs = min(s.values[0] for s in diag.values())
        for s in diag.values():
            s.shift = Egs
        allrel = np.sort(np.concatenate([s.values - s.shift for s in diag.values()]))
        cmap = cluster_mapping(allrel, p.fixeps)
        for s in diag.values():
            r = s.values - s.shift
            s.corr = np.array([cmap.get(float(x), float(x)) for x in r]) if cmap else r
        allcorr = np.sort(np.concatenate([s.corr for s in diag.values()]))
        Emax = highest_retained_energy(allcorr, p)
        keep_all = last and p.lastall
        for s in diag.values():
            s.nkept = len(s.values) if keep_all else int(np.count_nonzero(s.corr <= Emax))

        # after_diag (c++/core.hpp:193-230)
        res.td.append(self._td(N, diag))
        new_ops = None
        if p.strategy == "all":
            new_ops = self._recalc_singlets(diag, ops)
            res.custom.append(self._custom(N, diag, new_ops))
        for s in diag.values():
            s.nstored = s.nkept  # truncate_perform
        new_opch = opch if last else self._recalc_irreducible(diag)
        if p.strategy == "kept":
            new_ops = self._recalc_singlets(diag, ops)
            res.custom.append(self._custom(N, diag, new_ops))
        return diag, new_opch, new_ops

    def _assemble(self, ns: List[int], H: List[torch.Tensor], pieces: List[HPiece]) -> None:
        nb = len(ns)
        n = (C.c_int * nb)(*ns)
        Hp = (C.c_void_p * nb)(*[h.data_ptr() for h in H])
        arr = (HPiece * len(pieces))(*pieces)
        rc = self.ctx.lib.nrg_hamiltonian_batch(self.ctx.ptr, nb, n, Hp, len(pieces), arr, _stream_ptr(self.stream))
        if rc < 0:
            raise NRGError(rc, "nrg_hamiltonian_batch")

    def _recalc_irreducible(self, diag: Dict[Invar, Sub]) -> Dict[Tuple[Invar, Invar], torch.Tensor]:
        """SymmetryQS::recalc_irreduc with recalc_f (c++/recalc.hpp:52-76): <I1||f||Ip> over the
        kept states, one batched GEMM call for the whole step."""
        plan = []
        total = 0
        for Ip, sp in diag.items():
            for dq, table in qs.RECALC_F:
                I1 = (Ip[0] + dq[0], Ip[1] + dq[1])
                if I1 not in diag:
                    continue
                s1 = diag[I1]
                if not (s1.nstored and sp.nstored):
                    continue
                plan.append((I1, Ip, table, total))
                total += s1.nstored * sp.nstored
        buf = torch.zeros(max(total, 1), dtype=torch.float64, device=self.dev)
        out: Dict[Tuple[Invar, Invar], torch.Tensor] = {}
        terms = []
        for I1, Ip, table, off in plan:
            s1, sp = diag[I1], diag[Ip]
            f = buf[off:off + s1.nstored * sp.nstored].view(s1.nstored, sp.nstored)
            out[(I1, Ip)] = f
            for i1, ip, fn in table:
                A = s1.block(i1 - 1, s1.nstored)
                B = sp.block(ip - 1, sp.nstored)
                if A.shape[1] == 0 or B.shape[1] == 0:
                    continue
                terms.append(gemm3(f, fn(Ip[1]), A, None, B))
        if terms:
            gemm3_batch(terms, False, self.ctx, self.stream)
        return out

    def _recalc_singlets(self, diag: Dict[Invar, Sub], ops) -> Dict[str, Dict[Invar, torch.Tensor]]:
        """recalc_singlet (c++/symmetry.hpp:185-200) through recalc_general
        (c++/recalc.hpp:82-108) for every singlet operator over the stored states."""
        out: Dict[str, Dict[Invar, torch.Tensor]] = {}
        total = sum(len(ops) * s.nstored * s.nstored for s in diag.values())
        buf = torch.zeros(max(total, 1), dtype=torch.float64, device=self.dev)
        terms = []
        off = 0
        for name in sorted(ops):
            cold = ops[name]
            cnew = {}
            for I, s in diag.items():
                m = buf[off:off + s.nstored * s.nstored].view(s.nstored, s.nstored)
                off += s.nstored * s.nstored
                cnew[I] = m
                if s.nstored == 0:
                    continue
                for i, a in enumerate(qs.ancestors(I)):
                    if not qs.allowed(a) or a not in cold or s.dims[i] == 0:
                        continue
                    A = s.block(i, s.nstored)
                    O = cold[a][:s.dims[i], :s.dims[i]]  # trimmed to the kept ancestor states
                    terms.append(gemm3(m, 1.0, A, O, A))
            out[name] = cnew
        if terms:
            gemm3_batch(terms, False, self.ctx, self.stream)
        return out


def run_files(param_text: str, data_text: str, device: int = 0) -> Result:
    """Run the reference's ``param`` + ``data`` inputs; returns the td and custom rows."""
    kv = parse_param(param_text)
    if kv.get("symtype", "QS") != "QS":
        raise ValueError("symtype must be QS")
    return QSRun(RunParams.from_param(kv), read_data(data_text), device).run()
