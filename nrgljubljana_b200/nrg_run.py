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

from . import ddsum, qs
from ._lib import (GEMM3_DTYPE, HPIECE_DTYPE, NRG_HP_BLOCK, NRG_HP_DIAG, NRG_SPEC_DMNRG, NRG_SPEC_FDMGT,
                   NRG_SPEC_FDMLS, NRG_SPEC_FDMMATS, NRG_SPEC_FTMATS, SPECPAIR_DTYPE)
from .api import (BinGrid, Context, broaden, context, diag_batch_ptrs, gemm3_batch_array, hamiltonian_batch,
                  spec_accumulate_array, spec_accumulate_mats_array)
from .inputs import DataFile, SCALE, parse_param, read_data

Invar = Tuple[int, int]

# Parameters that do not change td/custom of a run without spectral functions.
_IGNORED = {
    "symtype", "model", "U", "Gamma", "delta", "band", "Tmin", "checksumrules", "logall", "log",
    "ops", "diag", "diagth",
    "Nmax",
    "variant", "spin", "Jkondo", "Jkondo1", "Jkondo2",
    # model parameters of the generated data and of its discretisation (keys of the data
    # generator, read by nrginit, not by the C++ run: c++/params.hpp has none of them)
    "U1", "U2", "Gamma1", "Gamma2", "eps1", "eps2", "U12", "J12", "tri", "mMAX", "smooth", "dos",
    "solpath", "xmax", "gamma", "options",
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
    # full-density-matrix algorithm (c++/params.hpp:240-253): FDM spectra (fdm: greater +
    # lesser parts, fdmgt/fdmls: each part alone), FDM expectation values at step fdmexpvn;
    # any of them keeps every state of the last step (params.hpp:535-539)
    fdm: bool = False
    fdmgt: bool = False
    fdmls: bool = False
    fdmmats: bool = False  # Green's functions on the Matsubara axis (c++/params.hpp:251-254)
    dmnrgmats: bool = False
    finitemats: bool = False
    mats: int = 100
    fdmexpv: bool = False
    fdmexpvn: int = 0
    lastalloverride: bool = False
    # complete-Fock-space spectra (c++/params.hpp:233-237): greater + lesser parts, or each alone
    cfs: bool = False
    cfsgt: bool = False
    cfsls: bool = False
    # conventional finite-temperature spectra (c++/params.hpp, "finite"; Algo_FT)
    finite: bool = False
    data_has_rescaled_energies: bool = True
    # DM-NRG spectra of the specs/specd/spect pairs (c++/params.hpp:181-396)
    T: float = 0.001
    dmnrg: bool = False
    specs: str = ""   # correlators of singlet operators
    specd: str = ""   # spectral functions of doublet operators
    spect: str = ""   # dynamic spin susceptibilities of triplet operators
    bins: int = 1000
    emin: float = -1.0
    emax: float = -1.0
    discard_immediately: float = 1e-16
    discard_trim: float = 1e-16
    goodE: float = 2.0
    NN1: bool = False
    NN2even: bool = True
    NN2avg: bool = False
    NNtanh: float = 0.0
    broaden: bool = True
    broaden_max: float = 10.0
    broaden_min: float = -99.0
    broaden_min_ratio: float = 3.0
    broaden_ratio: float = 1.05
    alpha: float = 0.3
    omega0: float = -1.0
    omega0_ratio: float = 1.0
    # output (c++/params.hpp:310, 332, 394-400): the raw trimmed bins as <name>.bin, a third
    # (imaginary) column, and the precision and width of the written numbers
    savebins: bool = False
    reim: bool = False
    # annotated.dat (c++/params.hpp:312-320): the lowest `dumpannotated` levels of every step
    dumpannotated: int = 0
    dumpprecision: int = 8
    dumpgroups: bool = True
    grouptol: float = 1e-6
    dumpscaled: bool = True
    dumpabs: bool = False
    dumpenergies: bool = False  # energies.nrg: every computed level of every step
    dumpsubspaces: bool = False  # subspaces.dat: kept and computed states of every subspace
    prec_td: int = 10
    prec_custom: int = 10
    prec_xy: int = 10
    width_td: int = 16
    width_custom: int = 16

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
        if (p.dmnrg or p.fdm_flags or p.cfs_flags) and p.strategy != "kept":
            raise ValueError("density-matrix algorithms are supported with strategy=kept")
        return p

    @property
    def fdm_flags(self) -> bool:
        """Params::fdm_flags (c++/params.hpp:535)."""
        return self.fdm or self.fdmgt or self.fdmls or self.fdmmats or self.fdmexpv

    @property
    def cfs_flags(self) -> bool:
        """Params::cfs_flags (c++/params.hpp:534)."""
        return self.cfs or self.cfsgt or self.cfsls

    @property
    def algorithms(self) -> List[str]:
        """The real-frequency spectral algorithms switched on (c++/oprecalc.hpp:123-131)."""
        return [a for a, on in (("DMNRG", self.dmnrg), ("FDM", self.fdm), ("FDMgt", self.fdmgt),
                                ("FDMls", self.fdmls), ("CFS", self.cfs), ("CFSgt", self.cfsgt),
                                ("CFSls", self.cfsls), ("FT", self.finite)) if on]

    @property
    def mats_algorithms(self) -> List[str]:
        """The Matsubara-axis algorithms switched on (c++/oprecalc.hpp:120-131)."""
        return [a for a, on in (("DMNRGmats", self.dmnrgmats), ("FDMmats", self.fdmmats),
                                ("FTmats", self.finitemats)) if on]

    @property
    def keep_all_states_in_last_step(self) -> bool:
        """Params::keep_all_states_in_last_step (c++/params.hpp:539)."""
        return self.lastall or ((self.cfs_flags or self.fdm_flags) and not self.lastalloverride)


@dataclass
class Result:
    td_fields: List[str]
    td: List[List[float]]
    custom_fields: List[str]
    custom: List[List[float]]
    blocks_per_step: List[int] = field(default_factory=list)
    max_dim_per_step: List[int] = field(default_factory=list)
    block_dims: List[List[int]] = field(default_factory=list)  # orders of the blocks of every step
    # file stem ("spec_DMNRG_dens_A_d-A_d", "corr_FDM_...", "spin_...") -> rows (E, A(E)),
    # the broadened spectra (broaden=true)
    spectra: Dict[str, np.ndarray] = field(default_factory=dict)
    # the same stems -> rows (E, Re w[, Im w]) of the trimmed raw bins (savebins=true)
    bins: Dict[str, np.ndarray] = field(default_factory=dict)
    annotated: List[str] = field(default_factory=list)  # lines of annotated.dat (dumpannotated > 0)
    energies: List[str] = field(default_factory=list)   # blocks of energies.nrg (dumpenergies)
    subspaces: List[str] = field(default_factory=list)  # lines of subspaces.dat (dumpsubspaces)
    tdfdm: Optional[Tuple[List[str], List[float]]] = None       # fields, row (fdm_thermodynamics)
    customfdm: Optional[Tuple[List[str], List[float]]] = None   # fields, row (measure_singlet_fdm)


# ------------------------------------------------------------------ host bookkeeping
def cluster_mapping(energies: np.ndarray, eps: float) -> Dict[float, float]:
    """Clusters(diag, epsilon) of c++/splitting.hpp:48-72 over the sorted energies: maps the
    members of a split cluster to its lowest value.

    The reference walks every value; a value whose gap to its predecessor is at least eps
    always starts a new cluster, so only the runs of smaller gaps need the walk, done here
    exactly as the reference does it. The reference's first cluster counts its first
    element twice (which changes nothing, a one-value cluster is never split) and the last
    cluster is never closed: a run that reaches the end of the list maps nothing for its
    last cluster."""
    mapping: Dict[float, float] = {}
    L = len(energies)
    if L < 2:
        return mapping
    small = np.diff(energies) < eps
    if not small.any():
        return mapping
    e = energies
    idx = np.flatnonzero(small)
    # runs of consecutive small gaps: elements a..b with gaps a..b-1 small
    brk = np.flatnonzero(np.diff(idx) > 1)
    starts = np.concatenate([[idx[0]], idx[brk + 1]])
    ends = np.concatenate([idx[brk], [idx[-1]]]) + 1
    # two-value runs (the common case: pairs split by round-off) in one pass; a pair is one
    # cluster, closed unless it ends the list
    pair = ends - starts == 1
    pa, pb = starts[pair], ends[pair]
    sel = (pb + 1 < L) & (e[pb] != e[pa])
    for x, y in zip(e[pb[sel]].tolist(), e[pa[sel]].tolist()):
        mapping.setdefault(x, y)
    for a, b in zip(starts[~pair].tolist(), ends[~pair].tolist()):
        run = e[a:b + 1].tolist()
        e0, i0 = run[0], 0
        for i in range(1, len(run) + 1):
            if i < len(run) and run[i] - e0 < eps:
                continue
            if i == len(run) and b + 1 >= L:
                break  # the last cluster of the list is never closed
            if i - i0 > 1:
                first = run[i0]
                if any(x != first for x in run[i0 + 1:i]):
                    for x in run[i0 + 1:i]:
                        if x != first:
                            mapping.setdefault(x, first)
            if i < len(run):
                e0, i0 = run[i], i
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
    """One subspace of a step: host eigenvalues and the address of its device eigenvectors."""
    I: Invar
    values: np.ndarray                 # computed eigenvalues (relative), ascending
    shift: float = 0.0
    corr: Optional[np.ndarray] = None  # corrected values (splitting fix), all computed
    nstored: int = 0                   # states kept after truncate_perform (all before)
    nkept: int = 0
    dims: List[int] = field(default_factory=list)  # ancestor block widths
    offs: List[int] = field(default_factory=list)  # their column offsets
    vptr: int = 0                      # device address of the n x n eigenvector rows
    n: int = 0


class MatSet:
    """Matrices of one kind in one flat device buffer, `nops` copies of the same layout
    (operator-major): the <||f||> of a step (nops = 1) or all singlet operators of a step.
    Keys map to (offset, rows, cols); every matrix is contiguous (ld = cols)."""

    def __init__(self, dev, shapes: Dict, nops: int = 1, host: Optional[np.ndarray] = None):
        self.loc: Dict = {}
        off = 0
        for k, (r, c) in shapes.items():
            self.loc[k] = (off, r, c)
            off += r * c
        self.total = off
        self.nops = nops
        if host is not None:
            self.buf = torch.from_numpy(host).to(dev)
        else:
            self.buf = torch.zeros(max(1, nops * off), dtype=torch.float64, device=dev)
        self.base = self.buf.data_ptr()

    def ptr(self, key, op: int = 0) -> int:
        return self.base + 8 * (op * self.total + self.loc[key][0])


def _pack(mats: List[Dict], shapes: Dict) -> np.ndarray:
    """Host image of a MatSet: for each dict in `mats` (one per operator) the matrices in
    the order of `shapes`; missing entries are zero."""
    total = sum(r * c for r, c in shapes.values())
    out = np.zeros(max(1, len(mats) * total))
    for o, m in enumerate(mats):
        off = o * total
        for k, (r, c) in shapes.items():
            if k in m:
                out[off:off + r * c] = np.ascontiguousarray(m[k], dtype=np.float64).ravel()
            off += r * c
    return out


@dataclass
class _Measure:
    """What one custom row needs, kept until the end of the run: the device diagonals of
    every singlet operator over the stored states, and the host Boltzmann weights."""
    T: float
    weights: np.ndarray        # mult(I) * exp(-f * corr) per stored state, subspace order
    diag: Optional[torch.Tensor]  # nops x states (device), gathered once the recalculation ran


@dataclass
class StepJob:
    """The blocks of one step of one run, assembled on the device and waiting for their
    eigensolve: orders, device addresses of H / eigenvalues / eigenvectors, the buffers
    that own them, and the subspace tasks in block order."""
    N: int
    tasks: list
    ns: List[int]
    Hp: List[int]
    Ep: List[int]
    Vp: List[int]
    Hbuf: torch.Tensor
    Ebuf: torch.Tensor
    Vbuf: torch.Tensor
    moff: np.ndarray
    voff: np.ndarray
    pcorr: torch.Tensor


@dataclass
class _StepRecord:
    """What the density-matrix sweeps and the spectral pass need of one step: its subspaces
    (all eigenvalues, kept counts, eigenvector locations), the eigenvectors, and
    Stats::total_energy after the step (the T_shift of its absolute energies)."""
    N: int
    scale: float
    diag: Dict[Invar, "Sub"]
    vecs: Optional[torch.Tensor]
    total_energy: float
    host: Optional[torch.Tensor] = None  # the eigenvectors while they are held in host memory
    base: int = 0                        # device address the subspaces' vptr point into

    def __post_init__(self):
        self.base = self.vecs.data_ptr() if self.vecs is not None else 0


class QSRun:
    """One NRG run (QS, one channel) on one device. ``run()`` does the whole run; a server
    drives ``start``, ``begin_step``, ``end_step`` and ``finish`` itself to solve the blocks
    of many runs in one batched call."""

    def __init__(self, params: RunParams, data: DataFile, device: int = 0, ctx: Optional[Context] = None):
        if data.symtype != "QS" or data.channels not in (1, 2):
            raise ValueError("the driver covers symtype QS with one or two channels")
        gnames = sorted(n for n, (k, _) in data.ops.items() if k == "g")
        known = qs.tables(data.channels).GLOBAL if data.channels in (1, 2) else {}
        if any(n not in known for n in gnames):
            # SymmetryQS::recalc_global knows Qdiff, Q1, Q2, Qtot of two channels and asserts
            # otherwise (c++/symmetry/nrg-recalc-QS.hpp:680-740)
            raise ValueError(f"global operators {[n for n in gnames if n not in known]}: QS has "
                             f"{sorted(known) or 'none'} with {data.channels} channel(s)")
        if data.nmax == 0 and params.algorithms:
            # Params::ZBW (Nmax = 0): the reference bins the initial cluster's spectra with its own
            # window rules (c++/spectrum.hpp:91-95); not restated here
            raise ValueError("zero-bandwidth runs (Nmax = 0) with spectral functions are not supported")
        self.T = qs.tables(data.channels)
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the QS run driver has no CPU fallback")
        self.p = params
        self.d = data
        self.dev = torch.device("cuda", device)
        self.ctx = ctx or context(device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.nmax = data.nmax
        self.sqrt_lambda = math.sqrt(params.Lambda)  # nrg_step_scale_factor (c++/params.hpp:639-641)
        # singlets, then global operators, each by name: the columns of `custom`
        # (singlet_operators_for_expv_evaluation, c++/output.hpp:121-127)
        self.gop_names = set(gnames)
        self.op_names = self._singlet_order(n for n, (k, _) in data.ops.items() if k in "sg")
        # (file prefix, kind, op1, op2) of the spectra (c++/oprecalc.hpp:160-195)
        self.algos = params.algorithms
        self.specs: List[Tuple[str, str, str, str]] = []
        if self.algos or params.mats_algorithms:
            for prefix, kind, text in (("corr", "s", params.specs), ("spec", "d", params.specd),
                                       ("spin", "t", params.spect)):
                for tok in text.split():
                    n1, n2 = tok.split("-", 1)
                    for name in (n1, n2):
                        k = data.ops.get(name, ("?",))[0]
                        if not (k == kind or (kind == "s" and k == "g")):
                            raise ValueError(f"{tok}: {name} is not a {dict(s='singlet', d='doublet', t='triplet')[kind]}"
                                             " operator of the data file")
                    self.specs.append((prefix, kind, n1, n2))
        self.dop_names = sorted({x for sp in self.specs if sp[1] == "d" for x in sp[2:]})
        self.top_names = sorted({x for sp in self.specs if sp[1] == "t" for x in sp[2:]})
        # singlets of the spectral pass: those of the correlators, and all of them for the FDM
        # expectation values
        self.sop_names = self._singlet_order({x for sp in self.specs if sp[1] == "s" for x in sp[2:]}
                                             | (set(self.op_names) if params.fdmexpv else set()))
        # the steps are kept (eigenvalues, eigenvectors, energy offsets) for the density
        # matrices and the spectral pass after the run
        self.keep_steps = bool(self.specs) or params.fdm_flags
        # A server merging the per-step recalculation of many runs sets these two lists: the
        # GEMM terms of end_step are then collected instead of launched, and the reads of
        # their outputs (the custom diagonals) wait in `deferred_reads` until the server has
        # launched all runs' terms in one nrg_gemm3_batch call.
        self.deferred_terms: Optional[List[np.ndarray]] = None
        self.deferred_reads: Optional[List] = None

    def _singlet_order(self, names) -> List[str]:
        names = set(names)
        return sorted(names - self.gop_names) + sorted(names & self.gop_names)

    def device_bytes(self) -> int:
        """Device bytes the run holds between steps: the current eigenvectors, the <||f||>
        and singlet-operator buffers, and the eigenvectors kept for the density matrices."""
        seen, total = set(), 0
        tensors = [getattr(self, "_vecs", None)]
        for name in ("opch", "ops"):
            m = getattr(self, name, None)
            tensors.append(m.buf if m is not None else None)
        tensors += [st.vecs for st in getattr(self, "dm_steps", []) if st.vecs is not None]
        for t in tensors:
            if t is not None and t.data_ptr() not in seen:
                seen.add(t.data_ptr())
                total += t.numel() * t.element_size()
        return total

    def _gemm(self, terms: np.ndarray, reads=()) -> None:
        """One batched GEMM call for `terms`, or their collection by a merging server. `reads`
        are the matrix sets the terms read besides this step's eigenvectors: collected terms
        keep them alive until the server's call is on the stream (the run drops its previous
        operators when the step ends, and the caching allocator may hand their memory to
        another run's outputs, whose zero fill would come first)."""
        if self.deferred_terms is not None:
            self.deferred_terms.append((terms, reads))
        else:
            gemm3_batch_array(terms, self.ctx, self.stream)

    # ---- scales (c++/step.hpp:30-39)
    def scale(self, trueN: int) -> float:
        return SCALE(trueN + 1, self.p.Lambda, self.p.discretization, self.p.z, self.p.bandrescale)

    def _h2d(self, a: np.ndarray) -> torch.Tensor:
        """Host array to the device without stalling the host: staged through pinned memory
        that the caching host allocator keeps until the copy on the stream has run."""
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().to(self.dev, non_blocking=True)

    # ---- measurements
    def _annotate(self, trueN: int, diag: Dict[Invar, Sub]) -> None:
        """perform_basic_measurements' annotated.dump (c++/measurements.hpp:229-233) over all
        computed states, before the truncation."""
        if self.p.dumpannotated > 0:
            entries = [(float(x), s.I) for s in diag.values() for x in (s.values - s.shift)]
            self.res.annotated += annotated_lines(entries, self.p, self.scale(trueN), self.total_energy)
        if self.p.dumpenergies:  # Output::dump_energies with the step index max(N, 0)
            self.res.energies.append(energies_block(max(trueN, 0), {s.I: s.values for s in diag.values()}))

    def _td(self, trueN: int, diag: Dict[Invar, Sub]) -> List[float]:
        """calculate_TD (c++/measurements.hpp:169-186) with SymmetryQS::calculate_TD."""
        f = self.p.betabar  # TD_factor (unscale = 1)
        subs = list(diag.values())
        counts = np.array([len(s.values) for s in subs])
        x = np.concatenate([s.values - s.shift for s in subs])
        m = np.repeat(np.array([qs.mult(s.I) for s in subs], dtype=np.float64), counts)
        ex = np.exp(-f * x)
        fx = f * x
        Z = float(np.sum(m * ex))
        E = float(np.sum(m * fx * ex))
        E2 = float(np.sum(m * fx * fx * ex))
        Zs = [qs.mult(s.I) * float(np.sum(np.exp(-f * s.corr[:s.nstored]))) for s in subs]
        T = self.scale(trueN) / self.p.betabar
        extra = qs.td_extra(Zs, [s.I for s in subs], Z)
        return [T] + extra + [E / Z, E2 / Z, E2 / Z - (E / Z) ** 2, -math.log(Z), E / Z + math.log(Z)]

    def _measure(self, trueN: int, diag: Dict[Invar, Sub], ops: MatSet) -> _Measure:
        """measure_singlet (c++/measurements.hpp:18-30): the diagonals are gathered on the
        device now and read back once at the end of the run."""
        f = self.p.betabar
        w, idx = [], []
        for s in diag.values():
            k = s.nstored
            w.append(qs.mult(s.I) * np.exp(-f * s.corr[:k]))
            off, r, c = ops.loc[s.I]
            idx.append(off + np.arange(k) * (c + 1))
        idx = np.concatenate(idx) if idx else np.zeros(0, dtype=np.int64)
        full = (np.arange(ops.nops)[:, None] * ops.total + idx[None, :]).ravel()
        g = self._h2d(full.astype(np.int64))
        m = _Measure(self.scale(trueN) / self.p.betabar, np.concatenate(w) if w else np.zeros(0), None)

        def gather():
            m.diag = torch.index_select(ops.buf, 0, g).view(ops.nops, len(idx))
        if self.deferred_reads is not None:
            self.deferred_reads.append(gather)
        else:
            gather()
        return m

    # ---- the run
    def start(self) -> None:
        """Initial subspaces, <||f||> and operators from the data file; docalc0
        (c++/core.hpp:251-260) measures them before the first step."""
        p, d = self.p, self.d
        scale0 = SCALE(0, p.Lambda, p.discretization, p.z, p.bandrescale)  # SCALE(Ninit)
        diag: Dict[Invar, Sub] = {}
        for I, e in sorted(d.subspaces):
            v = e.copy() if p.data_has_rescaled_energies else e / scale0
            diag[I] = Sub(I, v, 0.0, v.copy(), len(v), len(v), n=len(v))
        self.diag0 = diag  # the initial cluster, for the first run's spectra at N = -1 (Algo_FTmats)
        # <||f||> of every channel in one channel-major set; the keys each channel holds are
        # kept, as offdiag_function() needs its channel's matrix to exist
        ocs = [d.opch[ch][0] for ch in range(d.channels)]
        shapes = {}
        for oc in ocs:
            for k, m in oc.items():
                shapes[k] = m.shape
        self.opch = MatSet(self.dev, shapes, d.channels, _pack(ocs, shapes))
        self.opch_keys = [set(oc) for oc in ocs]
        mats = [{I1: m for (I1, I2), m in d.ops[name][1].items() if I1 == I2} for name in self.op_names]
        oshapes = {I: (s.nstored, s.nstored) for I, s in diag.items()}
        self.ops = MatSet(self.dev, oshapes, len(self.op_names), _pack(mats, oshapes))
        self.res = Result(["T"] + list(qs.TD_FIELDS) + ["<E>", "<E^2>", "C", "F", "S"], [], ["T"] + self.op_names,
                          [])
        self.meas: List[_Measure] = []
        self.dm_steps: List[_StepRecord] = []
        self.spilled_bytes = 0  # eigenvector bytes moved to host memory (and back) in this run
        self._kept_since_check = 0
        self.total_energy = float(d.gs_energy)  # Stats::total_energy (c++/stats.hpp:60-71)
        # operators of the spectral pass as read: singlets by subspace, doublets and triplets
        # by subspace pair
        self.spec_init: Dict[str, MatSet] = {}
        if self.sop_names:
            smats = [{I1: m for (I1, I2), m in d.ops[name][1].items() if I1 == I2} for name in self.sop_names]
            self.spec_init["s"] = MatSet(self.dev, oshapes, len(self.sop_names), _pack(smats, oshapes))
        for kind, names in (("d", self.dop_names), ("t", self.top_names)):
            if names:
                tmats = [dict(d.ops[name][1]) for name in names]
                tshapes = {}
                for m in tmats:
                    for k, mat in m.items():
                        tshapes[k] = mat.shape
                self.spec_init[kind] = MatSet(self.dev, tshapes, len(names), _pack(tmats, tshapes))
        if p.calc0:
            self._annotate(-1, diag)
            self.res.td.append(self._td(-1, diag))
            self.meas.append(self._measure(-1, diag, self.ops))
        # diag0 has identity eigenvectors: its <||f||> and operators are used as read.
        self.diag = diag
        self.N = 0

    @property
    def done(self) -> bool:
        return self.N >= self.nmax

    def run(self) -> Result:
        """The whole run on this device (nrg_loop, c++/core.hpp:286-293)."""
        self.start()
        while not self.done:
            job = self.begin_step()
            self.end_step(job, self._diagonalise(job))
        return self.finish()

    def finish(self) -> Result:
        """One device->host copy of all measured diagonals, then the custom rows."""
        res = self.res
        if self.meas:
            host = torch.cat([m.diag.reshape(-1) for m in self.meas]).cpu().numpy()
            k = 0
            for m in self.meas:
                nst = len(m.weights)
                dg = host[k:k + m.diag.numel()].reshape(len(self.op_names), nst)
                k += m.diag.numel()
                Z = float(np.sum(m.weights))
                res.custom.append([m.T] + [float(np.sum(m.weights * dg[o])) / Z for o in range(len(self.op_names))])
        self.meas = []
        if self.dm_steps:
            self._density_matrix_outputs(res)
            self.dm_steps = []
        return res

    def begin_step(self) -> "StepJob":
        """Subspace structure of step N and the assembly of its block Hamiltonians on the
        device; returns the blocks to diagonalise."""
        p, d = self.p, self.d
        N, prev, opch, res = self.N, self.diag, self.opch, self.res
        scale = self.scale(N)
        # subspace structure (c++/core.hpp:42-58, 62-70; c++/subspaces.hpp:114-121)
        new = set()
        for I in prev:
            for J in self.T.new_subspaces(I):
                if qs.allowed(J):
                    new.add(J)
        tasks: List[Tuple[Invar, List[int], List[Invar]]] = []
        for I in sorted(new):
            anc = self.T.ancestors(I)
            dims = [(prev[a].nstored if a in prev else 0) if qs.triangle(I, a, self.T.QN[i]) else 0
                    for i, a in enumerate(anc)]
            if sum(dims):
                tasks.append((I, dims, anc))
        nb = len(tasks)
        ns = [sum(t[1]) for t in tasks]
        res.blocks_per_step.append(nb)
        res.max_dim_per_step.append(max(ns))
        res.block_dims.append(ns)
        moff = np.zeros(nb + 1, dtype=np.int64)
        moff[1:] = np.cumsum(np.array(ns, dtype=np.int64) ** 2)
        voff = np.zeros(nb + 1, dtype=np.int64)
        voff[1:] = np.cumsum(ns)
        Hbuf = torch.empty(int(moff[-1]), dtype=torch.float64, device=self.dev)
        Vbuf = torch.empty(int(moff[-1]), dtype=torch.float64, device=self.dev)
        Ebuf = torch.empty(int(voff[-1]), dtype=torch.float64, device=self.dev)
        Hp = [Hbuf.data_ptr() + 8 * int(x) for x in moff[:-1]]
        Vp = [Vbuf.data_ptr() + 8 * int(x) for x in moff[:-1]]
        Ep = [Ebuf.data_ptr() + 8 * int(x) for x in voff[:-1]]

        # corrected ancestor energies on the device (one copy)
        poff, flat, o = {}, [], 0
        for I, s in prev.items():
            if s.nstored:
                poff[I] = o
                flat.append(s.corr[:s.nstored])
                o += s.nstored
        pcorr = self._h2d(np.concatenate(flat))
        pbase = pcorr.data_ptr()

        # Hamiltonian pieces: hamiltonian() + SymmetryQS::make_matrix
        rows = []
        xi, zeta = d.xi, d.zeta
        for b, (I, dims, anc) in enumerate(tasks):
            offs = [0] + np.cumsum(dims).tolist()[:-1]
            for i in range(self.T.COMBS):
                if dims[i]:
                    rows.append((b, NRG_HP_DIAG, offs[i], offs[i], dims[i], dims[i], 0, 0, 0,
                                 pbase + 8 * poff[anc[i]], self.sqrt_lambda, 0.0))
            ss = I[1]
            for (i, j, ch, fn) in self.T.OFFDIAG:
                if not (dims[i - 1] and dims[j - 1]):
                    continue
                factor = qs.ieee(fn, ss) * xi[ch][N]
                key = (anc[i - 1], anc[j - 1])
                if key not in self.opch_keys[ch]:
                    raise RuntimeError(f"offdiag_function(): matrix not found {i} {j} {ch} 0")
                _, r, c = opch.loc[key]
                if (r, c) != (dims[i - 1], dims[j - 1]):
                    raise AssertionError("qq.rmax(i-1) == size1(mat) && qq.rmax(j-1) == size2(mat)")
                fs = factor / scale
                if i > j:
                    rows.append((b, NRG_HP_BLOCK, offs[j - 1], offs[i - 1], dims[j - 1], dims[i - 1], 1, 0, c,
                                 opch.ptr(key, ch), fs, 0.0))
                else:
                    rows.append((b, NRG_HP_BLOCK, offs[i - 1], offs[j - 1], dims[i - 1], dims[j - 1], 0, 0, c,
                                 opch.ptr(key, ch), fs, 0.0))
            for (i, ch, number) in self.T.DIAG:
                if dims[i - 1]:
                    shift = zeta[ch][N + 1] * (number - 1.0 * qs.AVGOCCUP) / scale
                    rows.append((b, NRG_HP_DIAG, offs[i - 1], offs[i - 1], dims[i - 1], dims[i - 1], 0, 0, 0, 0,
                                 0.0, shift))
        hamiltonian_batch(ns, Hp, np.array(rows, dtype=HPIECE_DTYPE), self.ctx, self.stream)
        return StepJob(N, tasks, ns, Hp, Ep, Vp, Hbuf, Ebuf, Vbuf, moff, voff, pcorr)

    def end_step(self, job: "StepJob", info: np.ndarray) -> None:
        """do_diag and after_diag (c++/core.hpp:122-230) once the step's blocks are solved."""
        p = self.p
        N, tasks, ns, Vp, Ebuf, voff = job.N, job.tasks, job.ns, job.Vp, job.Ebuf, job.voff
        res, meas, opch, ops = self.res, self.meas, self.opch, self.ops
        last = N == self.nmax - 1
        if np.any(info != 0):
            b = int(np.nonzero(info)[0][0])
            raise RuntimeError(f"dsyev failed. INFO={int(info[b])} (subspace {tasks[b][0]})")
        evals = Ebuf.cpu().numpy()

        diag: Dict[Invar, Sub] = {}
        for b, (I, dims, anc) in enumerate(tasks):
            offs = [0] + np.cumsum(dims).tolist()[:-1]
            diag[I] = Sub(I, evals[voff[b]:voff[b + 1]], dims=list(dims), offs=offs, vptr=Vp[b], n=ns[b],
                          nstored=ns[b])
        # do_diag: Egs subtraction, splitting correction, truncation (c++/core.hpp:141-143)
        Egs = min(float(s.values[0]) for s in diag.values())  # Egs_subtraction (c++/eigen.hpp:321-333)
        self.total_energy += Egs * self.scale(N)  # Stats::update (c++/stats.hpp:65-71)
        for s in diag.values():
            s.shift = Egs
            s.corr = s.values - Egs
        allrel = np.sort(np.concatenate([s.corr for s in diag.values()]))
        cmap = cluster_mapping(allrel, p.fixeps)
        if cmap:  # Clusters::fix_it: every value found in the mapping is replaced
            keys = np.array(sorted(cmap))
            vals = np.array([cmap[k] for k in keys.tolist()])
            flat = np.concatenate([s.corr for s in diag.values()])
            pos = np.minimum(np.searchsorted(keys, flat), len(keys) - 1)
            hit = keys[pos] == flat
            flat = np.where(hit, vals[pos], flat)
            o = 0
            for s in diag.values():
                s.corr = flat[o:o + len(s.corr)]
                o += len(s.corr)
            allcorr = np.sort(flat)
        else:
            allcorr = allrel
        Emax = highest_retained_energy(allcorr, p)
        keep_all = last and p.keep_all_states_in_last_step
        for s in diag.values():
            s.nkept = len(s.values) if keep_all else int(np.count_nonzero(s.corr <= Emax))
        if p.dumpsubspaces:  # Store::dump_subspaces (c++/store.hpp:75-84), written after the run
            res.subspaces += [f"Iteration {N}", f"len_dm={len(diag)}"] + \
                [f"I={I[0]} {I[1]} kept={diag[I].nkept} total={len(diag[I].values)}" for I in sorted(diag)] + [""]

        # after_diag (c++/core.hpp:193-230)
        self._annotate(N, diag)
        res.td.append(self._td(N, diag))
        new_ops = ops
        if p.strategy == "all":
            new_ops = self._recalc_singlets(diag, ops, names=self.op_names)
            meas.append(self._measure(N, diag, new_ops))
        for s in diag.values():
            s.nstored = s.nkept  # truncate_perform
        new_opch = opch if last else self._recalc_irreducible(diag)
        if p.strategy == "kept":
            new_ops = self._recalc_singlets(diag, ops, names=self.op_names)
            meas.append(self._measure(N, diag, new_ops))
        self._vecs = job.Vbuf  # the step's eigenvectors stay allocated until the next step
        if self.keep_steps:  # the density matrices and spectra need every step's eigenvectors
            self.dm_steps.append(_StepRecord(N, self.scale(N), diag, job.Vbuf, self.total_energy))
            # the free memory is read (cudaMemGetInfo, milliseconds) once per GiB kept
            self._kept_since_check += 8 * int(job.moff[-1])
            if self._kept_since_check >= self.SPILL_CHECK_BYTES:
                self._kept_since_check = 0
                self._make_room(self.SPILL_HEADROOM_STEPS * 8 * int(job.moff[-1]),
                                range(len(self.dm_steps) - 1))
        self.diag, self.opch, self.ops = diag, new_opch, new_ops
        self.N = N + 1

    # A step whose blocks hold more than this many bytes gives the library's workspace back
    # after its eigensolve: the workspace arena only grows, and a run that keeps every step's
    # eigenvectors (spectra, FDM) needs that memory for its own later steps.
    TRIM_STEP_BYTES = 1 << 30

    # The kept steps' eigenvectors live on the device while it has room. When, after a step
    # (checked each time another SPILL_CHECK_BYTES of eigenvectors have been kept), the device
    # has less free memory than SPILL_HEADROOM_BYTES or SPILL_HEADROOM_STEPS times that step's
    # eigenvector bytes (the next step's matrices, eigenvectors and workspace come
    # out of it), the oldest steps move to pinned host memory; the density-matrix sweeps and
    # the spectral pass bring each step back when they reach it. This is the device form of
    # the reference's unitary files, DiagInfo::save / load (c++/eigen.hpp:389-413), which hold
    # every step's eigenvectors between the NRG run and the density-matrix pass.
    SPILL_HEADROOM_BYTES = 16 << 30
    SPILL_HEADROOM_STEPS = 6
    SPILL_CHECK_BYTES = 1 << 30

    def _free_device_bytes(self) -> int:
        free, _ = torch.cuda.mem_get_info(self.dev)
        return free + torch.cuda.memory_reserved(self.dev) - torch.cuda.memory_allocated(self.dev)

    def _make_room(self, need: int, candidates) -> None:
        """Gives the library's workspace back, then moves the eigenvectors of the steps in
        `candidates` (in that order) to host memory, until the device has
        max(need, SPILL_HEADROOM_BYTES) bytes free."""
        need = max(need, self.SPILL_HEADROOM_BYTES)
        free = self._free_device_bytes()
        if free >= need:
            return
        # first the memory that is only held for reuse: the library's workspace (it grows back
        # to what the next call needs) and torch's cache
        self.ctx.trim()
        torch.cuda.empty_cache()
        free = self._free_device_bytes()
        if free >= need:
            return
        for k in candidates:
            st = self.dm_steps[k]
            if st.vecs is None:
                continue
            host = torch.empty(st.vecs.shape, dtype=st.vecs.dtype, pin_memory=True)
            host.copy_(st.vecs)  # synchronous: the device buffer is free when this returns
            free += st.vecs.numel() * st.vecs.element_size()
            st.host, st.vecs = host, None
            self.spilled_bytes += host.numel() * host.element_size()
            if free >= need:
                break
        torch.cuda.empty_cache()  # the library's workspace is not allocated through torch

    def _resident(self, k: int, candidates) -> None:
        """Step k's eigenvectors on the device (moved back from host memory if they were
        spilled, the subspaces' addresses rebased); `candidates` give way first."""
        st = self.dm_steps[k]
        if st.vecs is not None:
            return
        nbytes = st.host.numel() * st.host.element_size()
        self._make_room(nbytes + self.SPILL_HEADROOM_STEPS * nbytes, [j for j in candidates if j != k])
        vecs = torch.empty(st.host.shape, dtype=st.host.dtype, device=self.dev)
        vecs.copy_(st.host)
        delta = vecs.data_ptr() - st.base
        for sub in st.diag.values():
            sub.vptr += delta
        st.vecs, st.base, st.host = vecs, vecs.data_ptr(), None

    def _diagonalise(self, job: "StepJob") -> np.ndarray:
        """All blocks of the step in one batched call (diagonalisations, c++/core.hpp:113-120)."""
        large = self.keep_steps and 16 * int(job.moff[-1]) > self.TRIM_STEP_BYTES
        if large and torch.cuda.memory_reserved(self.dev) - torch.cuda.memory_allocated(self.dev) > self.TRIM_STEP_BYTES:
            torch.cuda.empty_cache()  # memory cached by torch is out of the library's reach
        info = diag_batch_ptrs(job.ns, job.Hp, job.Ep, job.Vp, self.ctx, self.stream)
        if large:
            self.ctx.trim()
        return info

    def _recalc_irreducible(self, diag: Dict[Invar, Sub]) -> MatSet:
        """SymmetryQS::recalc_irreduc with recalc_f (c++/recalc.hpp:52-76): <I1||f_ch||Ip> of
        every channel over the kept states (channel-major), one batched GEMM call for the
        whole step. Every channel holds every pair of the plan."""
        plan = []
        dqs = []
        for dq, _, _ in self.T.RECALC_F:
            if dq not in dqs:
                dqs.append(dq)
        for Ip, sp in diag.items():
            for dq in dqs:
                I1 = (Ip[0] + dq[0], Ip[1] + dq[1])
                s1 = diag.get(I1)
                if s1 is None or not (s1.nstored and sp.nstored):
                    continue
                plan.append((I1, Ip))
        out = MatSet(self.dev, {(I1, Ip): (diag[I1].nstored, diag[Ip].nstored) for I1, Ip in plan},
                     self.T.channels)
        rows = []
        for I1, Ip in plan:
            s1, sp = diag[I1], diag[Ip]
            dq = (I1[0] - Ip[0], I1[1] - Ip[1])
            for tdq, ch, table in self.T.RECALC_F:
                if tdq != dq:
                    continue
                M = out.ptr((I1, Ip), ch)
                for i1, ip, fn in table:
                    k = s1.dims[i1 - 1]
                    if k == 0 or sp.dims[ip - 1] == 0:
                        continue
                    if k != sp.dims[ip - 1]:
                        raise AssertionError("size2(A) == size2(B)")  # product, c++/numerics_ublas.hpp:112
                    rows.append((M, sp.nstored, s1.vptr + 8 * s1.offs[i1 - 1], s1.n, 0, 0,
                                 sp.vptr + 8 * sp.offs[ip - 1], sp.n, s1.nstored, sp.nstored, k, k, 0, 1, qs.ieee(fn, Ip[1])))
        if rows:
            self._gemm(np.array(rows, dtype=GEMM3_DTYPE))
        self.opch_keys = [set(out.loc)] * self.T.channels
        return out

    def _recalc_singlets(self, diag: Dict[Invar, Sub], cold: MatSet, rows=None, names=()) -> MatSet:
        """recalc_singlet (c++/symmetry.hpp:185-200) through recalc_general
        (c++/recalc.hpp:82-108) for every singlet operator of `cold` over the stored states
        (or the first rows(s) states of each subspace): the terms of one operator are built
        once and replicated over the operators (operator-major). `names` are the operators of
        `cold` in its order; the global ones among them then gain the added site's charge,
        recalc_global / recalc1_global (c++/symmetry/nrg-recalc-QS.hpp:680-740,
        c++/recalc.hpp:111-122): <I||Q||I> += value * U_i1 U_ip^T over the same states, in the
        same batched call after the operator's recalc_general terms."""
        rows = rows or (lambda s: s.nstored)
        out = MatSet(self.dev, {I: (rows(s), rows(s)) for I, s in diag.items()}, cold.nops)
        base = []
        for I, s in diag.items():
            k = rows(s)
            if k == 0:
                continue
            M = out.ptr(I)
            for i, a in enumerate(self.T.ancestors(I)):
                w = s.dims[i]
                if w == 0 or not qs.allowed(a) or a not in cold.loc:
                    continue
                A = s.vptr + 8 * s.offs[i]
                _, r, c = cold.loc[a]
                base.append((M, k, A, s.n, cold.ptr(a), c, A, s.n, k, k, w, w, 0, 1, 1.0))
        if base and cold.nops:
            b = np.array(base, dtype=GEMM3_DTYPE)
            t = np.tile(b, cold.nops)
            op = np.repeat(np.arange(cold.nops, dtype=np.uint64), len(b))
            t["M"] += op * np.uint64(8 * out.total)
            t["O"] += op * np.uint64(8 * cold.total)
        else:
            t = np.zeros(0, dtype=GEMM3_DTYPE)
        glob = []
        for o, name in enumerate(names):
            if name not in self.gop_names:
                continue
            for I, s in diag.items():
                k = rows(s)
                if k == 0:
                    continue
                M = out.ptr(I, o)
                for i1, ip, _, value in self.T.GLOBAL[name]:
                    w = s.dims[i1 - 1]
                    if w == 0 or s.dims[ip - 1] == 0:
                        continue
                    glob.append((M, k, s.vptr + 8 * s.offs[i1 - 1], s.n, 0, 0, s.vptr + 8 * s.offs[ip - 1], s.n,
                                 k, k, w, s.dims[ip - 1], 0, 1, float(value)))
        if glob:
            t = np.concatenate([t, np.array(glob, dtype=GEMM3_DTYPE)])
        if len(t):
            self._gemm(t, (cold,))
        return out

    def _recalc_tensor(self, diag: Dict[Invar, Sub], cold: MatSet, tables, factor, rows=None) -> MatSet:
        """SymmetryQS::recalc_doublet / recalc_triplet (c++/symmetry/nrg-recalc-QS.hpp:32-117,
        495-640) through recalc_general (c++/recalc.hpp:82-108) over the kept states (or the
        first rows(s) states of each subspace), every operator of the set in one batched call
        (operator-major). `tables` lists (dq, rows) for Ip = I1 + dq; factor(fn, ss1)
        evaluates a row's coefficient."""
        rows = rows or (lambda s: s.nstored)
        plan = []
        for I1, s1 in diag.items():
            if not rows(s1):
                continue
            for dq, table in tables:
                Ip = (I1[0] + dq[0], I1[1] + dq[1])
                sp = diag.get(Ip)
                if sp is not None and rows(sp):
                    plan.append((I1, Ip, table))
        out = MatSet(self.dev, {(I1, Ip): (rows(diag[I1]), rows(diag[Ip])) for I1, Ip, _ in plan}, cold.nops)
        base = []
        for I1, Ip, table in plan:
            s1, sp = diag[I1], diag[Ip]
            anc1, ancp = self.T.ancestors(I1), self.T.ancestors(Ip)
            M = out.ptr((I1, Ip))
            for i1, ip, fn in table:
                IN1, INp = anc1[i1 - 1], ancp[ip - 1]
                if not (qs.allowed(IN1) and qs.allowed(INp)) or (IN1, INp) not in cold.loc:
                    continue
                w1, wp = s1.dims[i1 - 1], sp.dims[ip - 1]
                if w1 == 0 or wp == 0:
                    continue
                _, r, c = cold.loc[(IN1, INp)]
                base.append((M, rows(sp), s1.vptr + 8 * s1.offs[i1 - 1], s1.n, cold.ptr((IN1, INp)), c,
                             sp.vptr + 8 * sp.offs[ip - 1], sp.n, rows(s1), rows(sp), w1, wp, 0, 1,
                             factor(fn, I1[1])))
        if base:
            b = np.array(base, dtype=GEMM3_DTYPE)
            t = np.tile(b, cold.nops)
            op = np.repeat(np.arange(cold.nops, dtype=np.uint64), len(b))
            t["M"] += op * np.uint64(8 * out.total)
            t["O"] += op * np.uint64(8 * cold.total)
            gemm3_batch_array(t, self.ctx, self.stream)
        return out

    # ---- density matrices and spectra (the DMNRG run, c++/nrg-general.hpp:139-168)
    def _density_matrix_outputs(self, res: Result) -> None:
        """After the run: the DM-NRG density matrices (calc_rho), the FDM weights and density
        matrices with the FDM thermodynamics (calc_rhoFDM), then the spectral pass over the
        kept steps (the second run of the reference without its diagonalisations)."""
        p = self.p
        rhos = self._rho_dmnrg() if ("DMNRG" in self.algos or p.dmnrgmats or p.cfs_flags) else None  # need_rho
        fdm = self._rho_fdm() if p.fdm_flags else None
        if fdm is not None:
            res.tdfdm = (["T", "E_fdm", "C_fdm", "F_fdm", "S_fdm"], fdm["tdrow"])
        res.spectra, res.bins, expv = self._spectral_pass(rhos, fdm)
        if expv is not None:
            res.customfdm = (["T"] + self.sop_names, [p.T] + expv)

    def _sweep(self, rho_last: Optional[MatSet], diag_src) -> List[Optional[MatSet]]:
        """rho of step k-1 from rho of step k for k = last .. 1: the cdmI terms
        (c++/dmnrg.hpp:55-80) of calc_densitymatrix_iterN / calc_fulldensitymatrix_iterN
        (85-102, 165-197), all subspaces of a step in one batched call. rho_last: the dense
        density matrix of the last step (None: none); diag_src(k): None or (weights, loc)
        with loc[sub] = (offset, first state, count), a diagonal sector of step k's density
        matrix (the DD sector of FDM, or the whole last step), applied as U^T diag(w) U."""
        steps = self.dm_steps
        nst = len(steps)
        rhos: List[Optional[MatSet]] = [None] * nst
        rhos[nst - 1] = rho_last
        for k in range(nst - 1, 0, -1):
            self._resident(k, list(range(nst - 1, k, -1)) + list(range(0, k)))
            cur, prv = steps[k], steps[k - 1]
            out = MatSet(self.dev, {I: (s.nkept, s.nkept) for I, s in prv.diag.items()})
            dsrc = diag_src(k) if diag_src else None
            R = rhos[k]
            rows = []
            for I, sP in prv.diag.items():
                dim = sP.nkept
                if dim == 0:
                    continue
                for i, dl in enumerate(self.T.IN):
                    sub = (I[0] - dl[0], I[1] - dl[1])
                    sN = cur.diag.get(sub)
                    if sN is None or sN.dims[i] == 0:
                        continue
                    if sN.dims[i] != dim:
                        raise AssertionError("rmax == dim")  # cdmI, c++/dmnrg.hpp:73
                    coef = float(qs.mult(sub)) / float(qs.mult(I))
                    A = sN.vptr + 8 * sN.offs[i]
                    if R is not None and sub in R.loc and R.loc[sub][1]:
                        nw = R.loc[sub][1]
                        rows.append((out.ptr(I), dim, A, sN.n, R.ptr(sub), nw, A, sN.n, dim, dim, nw, nw, 1, 0, coef))
                    if dsrc is not None and sub in dsrc[1]:
                        off, r0, cnt = dsrc[1][sub]
                        if cnt:
                            Ad = A + 8 * r0 * sN.n
                            rows.append((out.ptr(I), dim, Ad, sN.n, dsrc[0].data_ptr() + 8 * off, 0, Ad, sN.n, dim,
                                         dim, cnt, cnt, 1, 0, coef))
            if rows:
                gemm3_batch_array(np.array(rows, dtype=GEMM3_DTYPE), self.ctx, self.stream)
            rhos[k - 1] = out
        return rhos

    def _traces(self, rhos: List[Optional[MatSet]]) -> List[float]:
        """Tr rho = sum_I mult(I) Tr rho_I of every step (one gather per step, one copy)."""
        diags, mults, counts = [], [], []
        for k, st in enumerate(self.dm_steps):
            R = rhos[k]
            idx, mv = [], []
            if R is not None:
                for I, (off, r, c) in R.loc.items():
                    idx.append(off + np.arange(r) * (c + 1))
                    mv.append(np.full(r, float(qs.mult(I))))
            ix = np.concatenate(idx).astype(np.int64) if idx else np.zeros(0, dtype=np.int64)
            counts.append(len(ix))
            mults.append(np.concatenate(mv) if mv else np.zeros(0))
            if len(ix):
                diags.append(torch.index_select(R.buf, 0, self._h2d(ix)))
        vals = torch.cat(diags).cpu().numpy() if diags else np.zeros(0)
        out, o = [], 0
        for cnt, mv in zip(counts, mults):
            out.append(float(np.sum(mv * vals[o:o + cnt])))
            o += cnt
        return out

    def _rho_dmnrg(self) -> List[Optional[MatSet]]:
        """init_rho over the kept states of the last step with scT = scale / T
        (c++/dmnrg.hpp:43-50) and the backward sweep; Tr rho = 1 at every step
        (check_trace_rho, c++/dmnrg.hpp:29-33)."""
        p = self.p
        last = self.dm_steps[-1]
        scT = last.scale / p.T
        Z = 0.0
        diagvals = {}
        for I, s in last.diag.items():
            ex = np.exp(-s.corr[:s.nkept] * scT)
            diagvals[I] = ex
            Z += qs.mult(I) * float(np.sum(ex))
        shapes = {I: (s.nkept, s.nkept) for I, s in last.diag.items()}
        host = np.zeros(max(1, sum(r * c for r, c in shapes.values())))
        o = 0
        for I, (r, c) in shapes.items():
            host[o + np.arange(r) * (c + 1)] = diagvals[I] / Z
            o += r * c
        self.Zft = Z  # calc_Z at the last step (c++/measurements.hpp:189-191): the same kept-state sum
        rhos = self._sweep(MatSet(self.dev, shapes, 1, host), None)
        for tr in self._traces(rhos):
            if abs(tr - 1.0) > 1e-9:
                raise RuntimeError(f"check_trace_rho() failed: {tr!r}")
        return rhos

    def _rho_fdm(self) -> Dict:
        """calc_ZnD and fdm_thermodynamics (c++/measurements.hpp:60-163) on the host in
        extended precision, init_rho_FDM (c++/dmnrg.hpp:146-162) and the FDM sweep
        (calc_fulldensitymatrix, 165-217) on the device: the KK sector as dense rotate terms,
        the DD sector of every step (and the whole last step) as diagonal ones."""
        p = self.p
        steps = self.dm_steps
        nst = len(steps)
        T = p.T
        GS = self.total_energy  # GS_energy = total_energy at the end (c++/nrg-general.hpp:133)
        combs = self.T.COMBS
        absz, mults, lo = [], [], []
        for k, st in enumerate(steps):
            last = k == nst - 1
            az, mu, l0 = {}, {}, {}
            for I, s in st.diag.items():
                az[I] = (s.values - s.shift) * st.scale  # Values::abs_zero (c++/eigen.hpp:45)
                mu[I] = float(qs.mult(I))
                l0[I] = 0 if last else s.nkept  # the D states, Sub::all() (c++/store.hpp:26-31)
            absz.append(az)
            mults.append(mu)
            lo.append(l0)
        ZG_terms, ZN_terms = [], []
        for k, st in enumerate(steps):
            g, n = [], []
            for I in st.diag:
                z = absz[k][I][lo[k][I]:]
                g.append(mults[k][I] * np.exp(-((z + st.total_energy) - GS) / T))  # abs_G (eigen.hpp:47)
                n.append(mults[k][I] * np.exp(-z / T))
            ZG_terms.append(np.concatenate(g) if g else np.zeros(0))
            ZN_terms.append(np.concatenate(n) if n else np.zeros(0))
        # ZZG = sum_N ZnDG[N] combs^(Nend-N-1); the powers are powers of two, so the scaled terms
        # are exact and one exactly rounded sum gives the 400-bit result rounded to double
        ZZG = math.fsum(np.concatenate([ZG_terms[k] * float(combs) ** (nst - k - 1) for k in range(nst)]))
        ZnDG = [math.fsum(ZG_terms[k]) for k in range(nst)]
        ZnDN = [ddsum.exact_sum([ZN_terms[k]]) for k in range(nst)]
        ZnDNd = [float(z) for z in ZnDN]
        wnfactor = [math.pow(combs, nst - k - 1) / ZZG for k in range(nst)]
        wn = [wnfactor[k] * ZnDG[k] for k in range(nst)]
        if abs(sum(wn) - 1.0) > 1e-12:
            raise RuntimeError(f"sum of w_n is {sum(wn)!r}, not 1")  # calc_ZnD sum rule
        # fdm_thermodynamics: E and E^2 moments over the D states of every shell
        from fractions import Fraction
        E = Fraction(0)
        E2 = Fraction(0)
        for k, st in enumerate(steps):
            if not wn[k] > 1e-16:
                continue
            dd, ee = [], []
            for I in st.diag:
                z = absz[k][I][lo[k][I]:]
                dd.append((wn[k] * mults[k][I]) * np.exp(-z / T))
                ee.append(z + st.total_energy)  # abs_T (eigen.hpp:46)
            d_ = np.concatenate(dd) if dd else np.zeros(0)
            e_ = np.concatenate(ee) if ee else np.zeros(0)
            E += ddsum.dot(d_, e_) / ZnDN[k]
            E2 += ddsum.dot_sq(d_, e_) / ZnDN[k]
        E_fdm = float(E)
        C_fdm = float(E2 - E * E) / math.pow(T, 2)
        F_fdm = -math.log(ZZG) * T + GS
        S_fdm = (E_fdm - F_fdm) / T
        # diagonal sectors of init_rho_FDM: exp(-E/T) w_n / Z_n^D over the D states
        dsrc = {}
        for k, st in enumerate(steps):
            loc, parts, o = {}, [], 0
            if ZnDNd[k] != 0.0 and wn[k] != 0.0:
                for I in st.diag:
                    w = (np.exp(-absz[k][I][lo[k][I]:] / T) * wn[k]) / ZnDNd[k]
                    loc[I] = (o, lo[k][I], len(w))
                    parts.append(w)
                    o += len(w)
            buf = self._h2d(np.concatenate(parts)) if parts else torch.zeros(1, dtype=torch.float64, device=self.dev)
            dsrc[k] = (buf, loc)
        rhos = self._sweep(None, lambda k: dsrc[k])
        traces = self._traces(rhos)
        for k in range(nst - 1):
            expected = sum(wn[k + 1:])
            if expected > 0 and abs((traces[k] - expected) / expected) > 1e-9:
                raise RuntimeError(f"Tr rhoFDM({k}) = {traces[k]!r}, expected {expected!r}")
        return {"rhos": rhos, "wn": wn, "wnfactor": wnfactor, "last": dsrc[nst - 1], "GS": GS,
                "tdrow": [T, E_fdm, C_fdm, F_fdm, S_fdm]}

    def _spectral_pass(self, rhos, fdm) -> Tuple[Dict[str, np.ndarray], Dict[str, np.ndarray], Optional[List[float]]]:
        """The spectra of the DMNRG run: per step the operators of the spectra recalculated
        (over all states when an FDM flag is set, do_recalc_all, c++/params.hpp:542-547;
        else over the kept ones), BaseSpectrum::calc over all subspace pairs
        (c++/algo.hpp:55-67) with Algo_DMNRG (c++/algo_DMNRG.hpp:29-52; merged with the
        N/N+2 or N/N+1 window, c++/spectrum.hpp:81-128) and Algo_FDMgt/ls
        (c++/algo_FDM.hpp:30-151; merged whole); the FDM expectation values at step
        fdmexpvn (c++/measurements.hpp:31-44, 218-221). At the end trim (c++/bins.hpp:165-185)
        and broaden on the device (c++/spectrum.hpp:168-196)."""
        p, d = self.p, self.d
        steps = self.dm_steps
        nst = len(steps)
        Lam = p.Lambda
        last_scale = SCALE(self.nmax, Lam, p.discretization, p.z, p.bandrescale)
        emax = p.emax if p.emax > 0 else SCALE(0, Lam, p.discretization, p.z, p.bandrescale) * 100.0
        emin = p.emin if p.emin > 0 else last_scale / 100.0
        grid = BinGrid.from_limits(emin, emax, p.bins, p.discard_immediately)
        ebins = grid.energies()
        nb = grid.nbins
        Efac = Lam if (d.channels == 1 and not p.NN1) else math.sqrt(Lam)  # Params::getEfactor
        # do_recalc_all (c++/params.hpp:542-547): the operators over all states for CFS and FDM
        rows = (lambda s: s.n) if (p.fdm_flags or p.cfs_flags) else (lambda s: s.nkept)  # noqa: E731
        kinds = {"s": (1, qs.correlator_factor, self.sop_names), "d": (-1, qs.specdens_factor, self.dop_names),
                 "t": (1, qs.dynamicsusceptibility_factor, self.top_names)}
        tables = {"d": (self.T.DOUBLET, self.T.doublet_factor), "t": (self.T.TRIPLET, qs.triplet_factor)}
        parts_of = {"FDM": ("gt", "ls"), "FDMgt": ("gt",), "FDMls": ("ls",)}
        fdm_parts = sorted({w for a in self.algos if a in parts_of for w in parts_of[a]})
        zeros = lambda: torch.zeros(nb, dtype=torch.float64, device=self.dev)  # noqa: E731
        dm_acc = {j: (np.zeros(nb), np.zeros(nb)) for j in range(len(self.specs))} if rhos is not None else {}
        fdm_acc = {(j, w): (zeros(), zeros()) for j in range(len(self.specs)) for w in fdm_parts}
        # the Matsubara algorithms: one GFMatsubara per spectrum, mats complex points
        # (c++/spectrum.hpp:212-227), every step's sums merged whole
        zm = lambda: torch.zeros(p.mats, dtype=torch.float64, device=self.dev)  # noqa: E731
        mats_acc = {(a, j): (zm(), zm()) for a in p.mats_algorithms for j in range(len(self.specs))}
        if "FTmats" in p.mats_algorithms and p.calc0 and self.specs:
            self._ftmats_initial(kinds, mats_acc)
        cfs_parts_of = {"CFS": ("gt", "ls"), "CFSgt": ("gt",), "CFSls": ("ls",)}
        cfs_parts = sorted({w for a in self.algos if a in cfs_parts_of for w in cfs_parts_of[a]})
        cfs_acc = {(j, w): (zeros(), zeros()) for j in range(len(self.specs)) for w in cfs_parts}
        ft_acc = {j: (np.zeros(nb), np.zeros(nb)) for j in range(len(self.specs))} if "FT" in self.algos else {}
        cur = dict(self.spec_init)
        expv = None
        for k, st in enumerate(steps):
            last = k == nst - 1
            if k:  # the pass is the last reader of the previous step's eigenvectors
                steps[k - 1].vecs = steps[k - 1].host = None
            self._resident(k, range(nst - 1, k, -1))
            cur = {kind: (self._recalc_singlets(st.diag, m, rows, self.sop_names) if kind == "s"
                          else self._recalc_tensor(st.diag, m, *tables[kind], rows)) for kind, m in cur.items()}
            dg = st.diag
            merge = p.NN1 or p.NN2avg or ((st.N % 2 == 0) if p.NN2even else (st.N % 2 == 1))
            if ("DMNRG" in self.algos and merge or p.dmnrgmats) and self.specs:
                rhoN = rhos[k]
                eoff, flat, o = {}, [], 0
                for I, s in dg.items():  # abs_zero energies of the kept states (c++/eigen.hpp:45)
                    eoff[I] = o
                    flat.append((s.values[:s.nkept] - s.shift) * st.scale)
                    o += s.nkept
                Edev = self._h2d(np.concatenate(flat) if flat else np.zeros(1))
                eb = Edev.data_ptr()
                Emin_w = st.scale * p.goodE
                Ex, Emax_w = Emin_w * Efac, Emin_w * Efac * Efac
                win = window(ebins, Emin_w, Ex, Emax_w, st.N == self.nmax - 1, st.N == 0, p.NNtanh)
                inside = (Emin_w < ebins) & (ebins < Emax_w)
                f = 0.5 if p.NN2avg else 1.0
                for j, (prefix, kind, n1, n2) in enumerate(self.specs):
                    sign, ff, names = kinds[kind]
                    ops = cur[kind]
                    o1, o2 = names.index(n1), names.index(n2)
                    pairs = []
                    for Ii, si in dg.items():
                        for Ij, sj in dg.items():
                            key = Ii if kind == "s" else (Ij, Ii)  # singlet sets are keyed by subspace
                            if (kind == "s" and Ij != Ii) or key not in ops.loc:
                                continue
                            ki, kj = si.nkept, sj.nkept
                            if ki == 0 or kj == 0:
                                continue
                            ld = ops.loc[key][2]
                            pairs.append((eb + 8 * eoff[Ii], eb + 8 * eoff[Ij], ops.ptr(key, o1), ld, ops.ptr(key, o2),
                                          ld, rhoN.ptr(Ii), ki, rhoN.ptr(Ij), kj, ki, ki, kj, kj, ki, kj, ff(Ii, Ij)))
                    if not pairs:
                        continue
                    if p.dmnrgmats:  # Algo_DMNRGmats::calc at every step (c++/algo_DMNRG.hpp:76-100)
                        re, im = mats_acc[("DMNRGmats", j)]
                        spec_accumulate_mats_array(NRG_SPEC_DMNRG, np.array(pairs, dtype=SPECPAIR_DTYPE), p.mats, re,
                                                   im, sign, p.T, 0.0, ctx=self.ctx, stream=self.stream)
                    if not ("DMNRG" in self.algos and merge):
                        continue
                    pos, neg = zeros(), zeros()
                    spec_accumulate_array(NRG_SPEC_DMNRG, np.array(pairs, dtype=SPECPAIR_DTYPE), grid, pos, neg,
                                          sign=sign, Emin=Emin_w, Emax=Emax_w, ctx=self.ctx, stream=self.stream)
                    for full, cs in zip(dm_acc[j], (pos.cpu().numpy(), neg.cpu().numpy())):
                        sel = inside & (cs != 0.0)  # mergeNN2half (c++/spectrum.hpp:114-128)
                        full[sel] += f * cs[sel] * win[sel]
            if (fdm_parts or p.fdmmats) and self.specs:
                GS = fdm["GS"]
                eoff, flat, o = {}, [], 0
                for I, s in dg.items():  # abs_G energies of all states (c++/eigen.hpp:47)
                    eoff[I] = o
                    flat.append(((s.values - s.shift) * st.scale + st.total_energy) - GS)
                    o += s.n
                Edev = self._h2d(np.concatenate(flat) if flat else np.zeros(1))
                eb = Edev.data_ptr()
                R = fdm["rhos"][k]
                for j, (prefix, kind, n1, n2) in enumerate(self.specs):
                    sign, ff, names = kinds[kind]
                    ops = cur[kind]
                    o1, o2 = names.index(n1), names.index(n2)
                    gt, ls, mt = [], [], []
                    for Ii, si in dg.items():
                        for Ij, sj in dg.items():
                            key = Ii if kind == "s" else (Ij, Ii)
                            if (kind == "s" and Ij != Ii) or key not in ops.loc:
                                continue
                            ni, nj = si.n, sj.n
                            Ki = 0 if last else si.nkept  # Eigen::boundary (c++/eigen.hpp:219-224)
                            Kj = 0 if last else sj.nkept
                            ld = ops.loc[key][2]
                            ri = R.ptr(Ii) if (R is not None and Ki) else 0
                            rj = R.ptr(Ij) if (R is not None and Kj) else 0
                            base = (eb + 8 * eoff[Ii], eb + 8 * eoff[Ij], ops.ptr(key, o1), ld, ops.ptr(key, o2), ld)
                            gt.append(base + (ri, max(Ki, 1), 0, 1, ni, Ki, nj, Kj, Ki, 0, ff(Ii, Ij)))
                            ls.append(base + (0, 1, rj, max(Kj, 1), ni, Ki, nj, Kj, 0, Kj, ff(Ii, Ij)))
                            mt.append(base + (ri, max(Ki, 1), rj, max(Kj, 1), ni, Ki, nj, Kj, Ki, Kj, ff(Ii, Ij)))
                    for w, prs, algo in (("gt", gt, NRG_SPEC_FDMGT), ("ls", ls, NRG_SPEC_FDMLS)):
                        if w in fdm_parts and prs:
                            pos, neg = fdm_acc[(j, w)]
                            spec_accumulate_array(algo, np.array(prs, dtype=SPECPAIR_DTYPE), grid, pos, neg,
                                                  sign=sign, T=p.T, wnf=fdm["wnfactor"][k], ctx=self.ctx,
                                                  stream=self.stream)
                    if p.fdmmats and mt:  # Algo_FDMmats::calc over the same pairs (c++/algo_FDM.hpp:167-217)
                        re, im = mats_acc[("FDMmats", j)]
                        spec_accumulate_mats_array(NRG_SPEC_FDMMATS, np.array(mt, dtype=SPECPAIR_DTYPE), p.mats, re, im,
                                                   sign, p.T, fdm["wnfactor"][k], ctx=self.ctx, stream=self.stream)
            if "FT" in self.algos and merge and self.specs:
                self._ft_step(st, cur, kinds, grid, ebins, Efac, ft_acc)
            if p.finitemats and self.specs:
                self._ftmats_step(st, cur, kinds, mats_acc)
            if cfs_parts and self.specs:
                self._cfs_step(st, last, None if last else rhos[k], cur, kinds, grid, cfs_parts, cfs_acc)
            if fdm is not None and p.fdmexpv and st.N == p.fdmexpvn:
                expv = self._fdm_expv(k, st, cur["s"], fdm)
        out: Dict[str, np.ndarray] = {}
        raw: Dict[str, np.ndarray] = {}
        for (a, j), (g_re, g_im) in mats_acc.items():  # GFMatsubara::save: w_n, Re, Im (c++/io.hpp:33-38)
            prefix, kind, n1, n2 = self.specs[j]
            sign = kinds[kind][0]
            wn = p.T * math.pi * (2 * np.arange(p.mats) + (0 if sign == 1 else 1))
            g_re, g_im = g_re.cpu().numpy(), g_im.cpu().numpy()
            g_im = np.where(np.abs(g_im) > np.abs(g_re) * 1e-10, g_im, 0.0)
            out[f"{prefix}_{a}_dens_{n1}-{n2}"] = np.stack([wn, g_re, g_im], axis=1)
        omega0 = p.omega0 if p.omega0 >= 0.0 else p.omega0_ratio * p.T
        bmin = p.broaden_min if p.broaden_min > 0.0 else p.broaden_min_ratio * last_scale
        mesh = []
        E = p.broaden_max
        while E > bmin:
            mesh.append(E)
            E /= p.broaden_ratio
        mesh = np.array(mesh)
        for j, (prefix, kind, n1, n2) in enumerate(self.specs):
            for a in self.algos:
                if a == "DMNRG":
                    full_pos, full_neg = dm_acc[j]
                elif a == "FT":
                    full_pos, full_neg = ft_acc[j]
                elif a in cfs_parts_of:
                    full_pos = sum(cfs_acc[(j, w)][0] for w in cfs_parts_of[a]).cpu().numpy()
                    full_neg = sum(cfs_acc[(j, w)][1] for w in cfs_parts_of[a]).cpu().numpy()
                else:
                    full_pos = sum(fdm_acc[(j, w)][0] for w in parts_of[a]).cpu().numpy()
                    full_neg = sum(fdm_acc[(j, w)][1] for w in parts_of[a]).cpu().numpy()
                name = f"{prefix}_{a}_dens_{n1}-{n2}"
                if p.broaden:
                    out[name] = self._broadened(full_pos, full_neg, ebins, mesh, omega0)
                if p.savebins:
                    raw[name] = raw_bins(full_pos, full_neg, ebins, p.discard_trim, p.reim)
        return out, raw, expv

    def _ftmats_add(self, dg: Dict[Invar, Sub], scale: float, cur: Dict, kinds: Dict, mats_acc: Dict) -> None:
        """Algo_FTmats::calc (c++/algo_FT.hpp:63-85) of one step for every spectrum: over
        kept(Ij) x kept(Ii), op1 op2 ((-sign) e^{-E1/T} + e^{-Ep/T}) / (Z_ft (i w_n - (E1 - Ep)))
        with the abs_zero energies and stats.Zft of the step (calc_Z, c++/measurements.hpp:
        189-191), one nrg_spec_accumulate_mats call per spectrum."""
        p = self.p
        scT = scale / p.T
        Z = sum(qs.mult(I) * float(np.sum(np.exp(-s.corr[:s.nkept] * scT))) for I, s in dg.items())
        eoff, flat, o = {}, [], 0
        for I, s in dg.items():  # abs_zero energies of the kept states (c++/eigen.hpp:45)
            eoff[I] = o
            flat.append((s.values[:s.nkept] - s.shift) * scale)
            o += s.nkept
        Edev = self._h2d(np.concatenate(flat) if flat else np.zeros(1))
        eb = Edev.data_ptr()
        for j, (prefix, kind, n1, n2) in enumerate(self.specs):
            sign, ff, names = kinds[kind]
            ops = cur[kind]
            o1, o2 = names.index(n1), names.index(n2)
            prs = []
            for Ii, si in dg.items():
                for Ij, sj in dg.items():
                    key = Ii if kind == "s" else (Ij, Ii)
                    if (kind == "s" and Ij != Ii) or key not in ops.loc:
                        continue
                    ki, kj = si.nkept, sj.nkept
                    if ki == 0 or kj == 0:
                        continue
                    ld = ops.loc[key][2]
                    prs.append((eb + 8 * eoff[Ii], eb + 8 * eoff[Ij], ops.ptr(key, o1), ld, ops.ptr(key, o2), ld,
                                0, 1, 0, 1, ki, 0, kj, 0, 0, 0, ff(Ii, Ij)))
            if prs:
                re, im = mats_acc[("FTmats", j)]
                spec_accumulate_mats_array(NRG_SPEC_FTMATS, np.array(prs, dtype=SPECPAIR_DTYPE), p.mats, re, im, sign,
                                           p.T, 1.0 / Z, ctx=self.ctx, stream=self.stream)

    def _ftmats_step(self, st: "_StepRecord", cur: Dict, kinds: Dict, mats_acc: Dict) -> None:
        self._ftmats_add(st.diag, st.scale, cur, kinds, mats_acc)

    def _ftmats_initial(self, kinds: Dict, mats_acc: Dict) -> None:
        """docalc0 runs the first run's spectral algorithms on the initial cluster as well
        (c++/core.hpp:251-260): the data file's eigenvalues with shift 0 and scale SCALE(Ninit),
        every state kept, the operators as read (c++/eigen.hpp:219-226, 314)."""
        self._ftmats_add(self.diag0, self.scale(-1), dict(self.spec_init), kinds, mats_acc)

    def _ft_step(self, st: "_StepRecord", cur: Dict, kinds: Dict, grid: BinGrid, ebins: np.ndarray, Efac: float,
                 ft_acc: Dict) -> None:
        """Algo_FT::calc (c++/algo_FT.hpp:28-43) of one step for every spectrum: over kept(Ij) x
        kept(Ii), op1 op2 ((-sign) e^{-E1/T} + e^{-Ep/T}) / Z_ft at E1 - Ep, with the abs_zero
        energies and stats.Zft of this step (calc_Z, c++/measurements.hpp:189-191). The two
        exponentials are the FDMls and the FDMgt D x D terms of the pair cut to its kept states
        (K = 0) with wnf = 1/Z_ft, accumulated into one bin set; the step's bins are then merged
        with the N/N+2 window (mergeNN2half, c++/spectrum.hpp:114-128) as for DMNRG."""
        p = self.p
        dg = st.diag
        scT = st.scale / p.T
        Z = sum(qs.mult(I) * float(np.sum(np.exp(-s.corr[:s.nkept] * scT))) for I, s in dg.items())
        eoff, flat, o = {}, [], 0
        for I, s in dg.items():  # abs_zero energies of the kept states (c++/eigen.hpp:45)
            eoff[I] = o
            flat.append((s.values[:s.nkept] - s.shift) * st.scale)
            o += s.nkept
        Edev = self._h2d(np.concatenate(flat) if flat else np.zeros(1))
        eb = Edev.data_ptr()
        Emin_w = st.scale * p.goodE
        Ex, Emax_w = Emin_w * Efac, Emin_w * Efac * Efac
        win = window(ebins, Emin_w, Ex, Emax_w, st.N == self.nmax - 1, st.N == 0, p.NNtanh)
        inside = (Emin_w < ebins) & (ebins < Emax_w)
        f = 0.5 if p.NN2avg else 1.0
        for j, (prefix, kind, n1, n2) in enumerate(self.specs):
            sign, ff, names = kinds[kind]
            ops = cur[kind]
            o1, o2 = names.index(n1), names.index(n2)
            prs = []
            for Ii, si in dg.items():
                for Ij, sj in dg.items():
                    key = Ii if kind == "s" else (Ij, Ii)
                    if (kind == "s" and Ij != Ii) or key not in ops.loc:
                        continue
                    ki, kj = si.nkept, sj.nkept
                    if ki == 0 or kj == 0:
                        continue
                    ld = ops.loc[key][2]
                    prs.append((eb + 8 * eoff[Ii], eb + 8 * eoff[Ij], ops.ptr(key, o1), ld, ops.ptr(key, o2), ld,
                                0, 1, 0, 1, ki, 0, kj, 0, 0, 0, ff(Ii, Ij)))
            if not prs:
                continue
            arr = np.array(prs, dtype=SPECPAIR_DTYPE)
            pos = torch.zeros(grid.nbins, dtype=torch.float64, device=self.dev)
            neg = torch.zeros(grid.nbins, dtype=torch.float64, device=self.dev)
            for algo in (NRG_SPEC_FDMGT, NRG_SPEC_FDMLS):
                spec_accumulate_array(algo, arr, grid, pos, neg, sign=sign, T=p.T, wnf=1.0 / Z, ctx=self.ctx,
                                      stream=self.stream)
            for full, cs in zip(ft_acc[j], (pos.cpu().numpy(), neg.cpu().numpy())):
                sel = inside & (cs != 0.0)
                full[sel] += f * cs[sel] * win[sel]

    def _cfs_step(self, st: "_StepRecord", last: bool, rhoN: Optional[MatSet], cur: Dict, kinds: Dict,
                  grid: BinGrid, cfs_parts: List[str], cfs_acc: Dict) -> None:
        """Algo_CFSgt / Algo_CFSls::calc (c++/algo_CFS.hpp:28-53, 80-105) of one step for every
        spectrum, merged whole (mergeCFS), built from the FDM pair modes of nrg_spec_accumulate
        with the abs_zero energies of all states (c++/eigen.hpp:45) and the DM-NRG rho:
          last step: the kept x kept term e^{-E/T}/Z_ft is the FDMgt (greater) and FDMls
            (lesser) D x D term of the pair cut to its kept states (K = 0) with wnf = 1/Z_ft;
          other steps: CFSls, sum over discarded(Ij) x kept(Ii) of op1 (op2 rho(Ii)) (-sign), is
            the FDMgt K(Ii) x D(Ij) term with rho(Ii); CFSgt, over kept(Ij) x discarded(Ii) of
            (op1^T rho(Ij))^T op2, is the FDMls D(Ii) x K(Ij) term with the operators swapped
            and rho(Ij) (rho is symmetric); both with wnf = 0, which zeroes the other FDM
            terms, and the factor times -sign, which cancels or supplies the FDM sign."""
        p = self.p
        dg = st.diag
        eoff, flat, o = {}, [], 0
        for I, s in dg.items():
            eoff[I] = o
            flat.append((s.values - s.shift) * st.scale)
            o += s.n
        Edev = self._h2d(np.concatenate(flat) if flat else np.zeros(1))
        eb = Edev.data_ptr()
        for j, (prefix, kind, n1, n2) in enumerate(self.specs):
            sign, ff, names = kinds[kind]
            ops = cur[kind]
            o1, o2 = names.index(n1), names.index(n2)
            gt, ls = [], []
            for Ii, si in dg.items():
                for Ij, sj in dg.items():
                    key = Ii if kind == "s" else (Ij, Ii)
                    if (kind == "s" and Ij != Ii) or key not in ops.loc:
                        continue
                    ld = ops.loc[key][2]
                    ki, kj, ni, nj = si.nkept, sj.nkept, si.n, sj.n
                    Ep_i, Ep_j, p1, p2, f = eb + 8 * eoff[Ii], eb + 8 * eoff[Ij], ops.ptr(key, o1), ops.ptr(key, o2), ff(Ii, Ij)
                    if last:
                        if ki and kj:
                            row = (Ep_i, Ep_j, p1, ld, p2, ld, 0, 1, 0, 1, ki, 0, kj, 0, 0, 0, f)
                            gt.append(row)
                            ls.append(row)
                    else:
                        if ki and nj > kj:
                            ls.append((Ep_i, Ep_j, p1, ld, p2, ld, rhoN.ptr(Ii), ki, 0, 1, ni, ki, nj, kj, ki, 0,
                                       -sign * f))
                        if kj and ni > ki:
                            gt.append((Ep_i, Ep_j, p2, ld, p1, ld, 0, 1, rhoN.ptr(Ij), kj, ni, ki, nj, kj, 0, kj,
                                       -sign * f))
            if last:
                calls = (("gt", gt, NRG_SPEC_FDMGT), ("ls", ls, NRG_SPEC_FDMLS))
                wnf = 1.0 / self.Zft
            else:
                calls = (("gt", gt, NRG_SPEC_FDMLS), ("ls", ls, NRG_SPEC_FDMGT))
                wnf = 0.0
            for w, prs, algo in calls:
                if w in cfs_parts and prs:
                    pos, neg = cfs_acc[(j, w)]
                    spec_accumulate_array(algo, np.array(prs, dtype=SPECPAIR_DTYPE), grid, pos, neg, sign=sign,
                                          T=p.T, wnf=wnf, ctx=self.ctx, stream=self.stream)

    def _fdm_expv(self, k: int, st: "_StepRecord", sops: MatSet, fdm: Dict) -> List[float]:
        """measure_singlet_fdm (c++/measurements.hpp:31-44): sum_I mult(I) Tr[rhoFDM_I O_I] over
        the kept states of step k, for every singlet operator."""
        R = fdm["rhos"][k]
        vals = []
        for o, name in enumerate(self.sop_names):
            acc = torch.zeros((), dtype=torch.float64, device=self.dev)
            for I, s in st.diag.items():
                kk = s.nkept
                if kk == 0 or I not in sops.loc:
                    continue
                off, r, c = sops.loc[I]
                Om = sops.buf[o * sops.total + off: o * sops.total + off + r * c].view(r, c)[:kk, :kk]
                if R is not None:  # dense KK density matrix
                    roff, rr, rc = R.loc[I]
                    Rm = R.buf[roff: roff + rr * rc].view(rr, rc)[:kk, :kk]
                    acc = acc + qs.mult(I) * torch.sum(Rm * Om.T)
                else:  # the last step: the diagonal init_rho_FDM
                    buf, loc = fdm["last"]
                    if I in loc:
                        woff, r0, cnt = loc[I]
                        acc = acc + qs.mult(I) * torch.sum(buf[woff: woff + kk] * torch.diagonal(Om))
            vals.append(acc)
        return [float(v) for v in torch.stack(vals).cpu().numpy()] if vals else []

    def _broadened(self, full_pos: np.ndarray, full_neg: np.ndarray, ebins: np.ndarray, mesh: np.ndarray,
                   omega0: float) -> np.ndarray:
        """Bins::trim (c++/bins.hpp:165-185) of both halves, then SpectrumRealFreq::continuous
        (c++/spectrum.hpp:168-196) on the device; rows (E, A(E)) sorted by E."""
        p = self.p

        ep, wp = trim_bins(ebins, full_pos, p.discard_trim)
        en, wn = trim_bins(ebins, full_neg, p.discard_trim)
        spikes_e = np.concatenate([ep, -en])
        spikes_w = np.concatenate([wp, wn])
        mesh_all = np.concatenate([mesh, -mesh])
        vals = broaden(spikes_e, spikes_w, mesh_all, p.alpha, omega0, self.ctx, self.stream)
        npos = len(mesh)
        rows_pos = sorted(zip(mesh_all[:npos].tolist(), vals[:npos].tolist()))
        rows_neg = sorted(zip(mesh_all[npos:].tolist(), vals[npos:].tolist()))
        return np.array(rows_neg + rows_pos)

def my_fcmp(x: float, y: float, eps: float) -> int:
    """my_fcmp (c++/numerics.hpp:107-114) with one epsilon: 0 when x and y are both zero, both
    below eps in magnitude, or closer than eps * (|x| + |y|); else the sign of x - y."""
    if (x == 0.0 and y == 0.0) or (abs(x) < eps and abs(y) < eps) or abs(x - y) < eps * (abs(x) + abs(y)):
        return 0
    return 1 if x > y else -1


def annotated_lines(entries: List[Tuple[float, Invar]], p: "RunParams", scale: float, total_energy: float) -> List[str]:
    """Annotated::dump (c++/output.hpp:77-125) for one step: `entries` are (energy relative to
    the step's ground state, subspace) of all computed states. The lowest p.dumpannotated of
    them, extended while the next one is within p.grouptol of the last (a cluster is dumped
    whole), one line per group of levels within p.grouptol of its first, "E (Q SS) ...
    [multiplicity]" with the labels sorted as strings (dumpgroups), or one line "E Q SS" per
    level; E in units of the step (dumpscaled) or times `scale`, plus `total_energy` with
    dumpabs; a blank line ends the step."""
    lst = sorted(entries)
    n = min(len(lst), p.dumpannotated)
    while n < len(lst) - 1 and my_fcmp(lst[n][0], lst[n - 1][0], p.grouptol) == 0:
        n += 1

    def num(x: float) -> str:
        return f"{x * (1.0 if p.dumpscaled else scale) + (total_energy if p.dumpabs else 0.0):.{p.dumpprecision}g}"
    out = []
    if p.dumpgroups:
        i = 0
        while i < n:
            e0 = lst[i][0]
            labels, deg = [], 0
            while i < n and my_fcmp(lst[i][0], e0, p.grouptol) == 0:
                I = lst[i][1]
                labels.append(f"{I[0]} {I[1]}")
                deg += qs.mult(I)
                i += 1
            out.append(num(e0) + "".join(f" ({q})" for q in sorted(labels)) + f" [{deg}]")
    else:
        out.extend(f"{num(e)} {I[0]} {I[1]}" for e, I in lst[:n])
    out.append("")
    return out


def energies_block(label: int, levels: Dict[Invar, np.ndarray]) -> str:
    """Output::dump_energies (c++/output.hpp:157-161) with DiagInfo::dump_energies
    (c++/eigen.hpp:349-352): "===== Iteration number: <label>" after a blank line, then every
    subspace in order, "Subspace: Q SS" and its raw eigenvalues (Values::all_rel, the
    ground-state shift not subtracted), each followed by a space, in the default 6-digit form
    of a C++ stream."""
    text = f"\n===== Iteration number: {label}\n"
    for I in sorted(levels):
        text += f"Subspace: {I[0]} {I[1]}\n" + "".join(f"{x:g} " for x in levels[I]) + "\n"
    return text


def trim_bins(ebins: np.ndarray, w: np.ndarray, discard_trim: float) -> Tuple[np.ndarray, np.ndarray]:
    """Bins::trim (c++/bins.hpp:165-185) of one half: bin i (energy ebins[i], weight w[i]) is
    kept if |w[i]| >= discard_trim * (ebins[i+1] - ebins[i]); the last bin is always kept."""
    width = np.diff(ebins)
    keep = np.concatenate([np.abs(w[:-1]) >= discard_trim * width, [True]])
    return ebins[keep], w[keep]


def raw_bins(full_pos: np.ndarray, full_neg: np.ndarray, ebins: np.ndarray, discard_trim: float,
             reim: bool = False) -> np.ndarray:
    """SpectrumRealFreq::savebins (c++/spectrum.hpp:146-170) after the trim of both halves:
    rows (E, Re w) -- (E, Re w, Im w) with reim -- of the kept positive-energy bins by ascending
    E, then of the kept negative-energy bins by ascending |E|, with E = -|E|. The weights of
    these real runs have no imaginary part, written as 0."""
    ep, wp = trim_bins(ebins, full_pos, discard_trim)
    en, wn = trim_bins(ebins, full_neg, discard_trim)
    cols = [np.concatenate([ep, -en]), np.concatenate([wp, wn])]
    if reim:
        cols.append(np.zeros(len(cols[0])))
    return np.stack(cols, axis=1)


def write_bins(path: str, rows: np.ndarray) -> None:
    """The binary file of savebins: the rows' doubles in order, native byte order, no header."""
    np.ascontiguousarray(rows, dtype=np.float64).tofile(path)


def window(e: np.ndarray, Emin: float, Ex: float, Emax: float, last: bool, first: bool, NNtanh: float) -> np.ndarray:
    """windowfunction (c++/spectrum.hpp:91-109) for the bin energies inside (Emin, Emax)."""
    def fnc(x):
        if NNtanh > 0:
            t0 = lambda y: np.tanh(NNtanh * (y - 0.5))  # noqa: E731
            return (t0(x) - t0(0.0)) / (t0(1.0) - t0(0.0))
        return x
    f = np.zeros_like(e)
    lo = (Emin < e) & (e <= Ex)
    hi = (Ex < e) & (e < Emax)
    f[lo] = fnc((e[lo] - Emin) / (Ex - Emin))
    f[hi] = 1.0 - fnc((e[hi] - Ex) / (Emax - Ex))
    if first:
        f[e >= Ex] = 1.0
    if last:
        f[e <= Ex] = 1.0
    return f


def run_files(param_text: str, data_text: str, device: int = 0) -> Result:
    """Run the reference's ``param`` + ``data`` inputs; returns the td and custom rows."""
    kv = parse_param(param_text)
    if kv.get("symtype", "QS") != "QS":
        raise ValueError("symtype must be QS")
    return QSRun(RunParams.from_param(kv), read_data(data_text), device).run()


def _write_table(path: str, fields: List[str], rows: List[List[float]], prec: int = 10, width: int = 16) -> None:
    """Columns as the reference's td/custom files print them (c++/outfield.hpp)."""
    with open(path, "w") as f:
        f.write("#" + "".join(f"{k:>{width}} " for k in fields).rstrip(" ") + " \n")
        for r in rows:
            f.write(" " + "".join(f"{v:>{width}.{prec}g} " for v in r) + "\n")


def main(argv=None) -> int:
    """python -m nrgljubljana_b200.nrg_run DIR [--out OUT] [--repeat K]: run DIR/param with
    DIR/data on the GPU and write OUT/td and OUT/custom (default OUT = DIR)."""
    import argparse
    import os
    import time
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("dir")
    ap.add_argument("--out", default=None)
    ap.add_argument("--repeat", type=int, default=1, help="run K times (timing); the last run is written")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    param = open(os.path.join(a.dir, "param")).read()
    data = open(os.path.join(a.dir, "data")).read()
    kv = parse_param(param)
    p, d = RunParams.from_param(kv), read_data(data)
    res = None
    for k in range(max(1, a.repeat)):
        t0 = time.perf_counter()
        res = QSRun(p, d, a.device).run()
        torch.cuda.synchronize()
        print(f"run {k}: {d.nmax} steps in {time.perf_counter() - t0:.3f} s", flush=True)
    out = a.out or a.dir
    write_outputs(out, p, res)
    return 0


def write_outputs(out: str, p: RunParams, res: Result) -> None:
    """td, custom, tdfdm, customfdm, the broadened spectra <stem>.dat (as Spikes::save and
    outputxy write them, c++/spectral.hpp:24-30, c++/io.hpp:33-38) and the raw bins <stem>.bin
    into the folder `out`."""
    import os
    os.makedirs(out, exist_ok=True)
    _write_table(os.path.join(out, "td"), res.td_fields, res.td, p.prec_td, p.width_td)
    _write_table(os.path.join(out, "custom"), res.custom_fields, res.custom, p.prec_custom, p.width_custom)
    for name, tab, prec, width in (("tdfdm", res.tdfdm, p.prec_td, p.width_td),
                                   ("customfdm", res.customfdm, p.prec_custom, p.width_custom)):
        if tab is not None:
            _write_table(os.path.join(out, name), tab[0], [tab[1]], prec, width)
    for name, rows in res.spectra.items():  # <prefix>_<algo>_dens_<op1>-<op2>.dat
        with open(os.path.join(out, f"{name}.dat"), "w") as f:
            for row in rows:  # (E, A(E)), or (w_n, Re G, Im G) on the Matsubara axis
                f.write(" ".join(f"{x:.{p.prec_xy}g}" for x in row) + (" 0\n" if p.reim and len(row) == 2 else "\n"))
    for name, rows in res.bins.items():
        write_bins(os.path.join(out, f"{name}.bin"), rows)
    if p.dumpsubspaces:
        with open(os.path.join(out, "subspaces.dat"), "w") as f:
            f.write("".join(line + "\n" for line in res.subspaces))
    if p.dumpenergies:
        with open(os.path.join(out, "energies.nrg"), "w") as f:
            f.write("".join(res.energies))
    if p.dumpannotated > 0:
        with open(os.path.join(out, "annotated.dat"), "w") as f:
            f.write("\n".join(res.annotated) + ("\n" if res.annotated else ""))


if __name__ == "__main__":
    raise SystemExit(main())
