"""Serving loop: many independent NRG runs on one device, continuously batched.

Requests (a ``param`` + ``data`` pair each, with an arrival time) are admitted while the
device-memory budget and the slot limit allow; every tick, each active run builds and
assembles its next step (``QSRun.begin_step``), the blocks of all active runs are solved in
ONE ``nrg_diag_batch`` call, each run finishes its step on the host (truncation,
thermodynamics; ``QSRun.end_step``) while its recalculation terms (the <||f||> of the next
Hamiltonian and the singlet operators, c++/oprecalc.hpp:71-87, 205-221) are collected, and
the terms of all active runs go to the device in ONE ``nrg_gemm3_batch`` call. Runs join and
leave the batch between ticks, so a request that arrives while others are on the GPU starts
at the next tick and overlaps their work. Every run's matrices stay resident in device
memory for its whole life; a run is charged at admission what it will hold (every step's
eigenvectors when it computes spectra or FDM quantities) and, once running, the larger of
that charge and what it actually holds.

Each block is solved by the same kernels whatever else is in the batch, so a run's result
does not depend on the mix it was served in.

There is no counterpart in the reference (one ``nrg`` process per run); this is the
serving pattern for z-averaging, parameter sweeps and request streams.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from .api import context, diag_batch_ptrs, gemm3_batch_array
from .inputs import parse_param, read_data
from .nrg_run import QSRun, Result, RunParams


@dataclass
class Request:
    rid: int
    param: str
    data: str
    arrival: float = 0.0  # seconds after the start of the stream
    tag: str = ""


@dataclass
class Completed:
    rid: int
    tag: str
    result: Result
    arrival: float
    admitted: float
    done: float
    steps: int

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def run_bytes(p: RunParams, nmax: int = 0, channels: int = 1) -> int:
    """Device bytes a run is charged at admission. One step holds its Hamiltonians, its
    eigenvectors and the previous step's eigenvectors, 3 x 8 B x sum of n^2, bounded by the
    kept states spread over at least four (Q, S) sectors of 4^channels x keep states each. A
    run whose density matrices or spectra need every step's eigenvectors after the forward
    sweep (any spectral algorithm, or FDM) keeps one more step's worth per step (nmax)."""
    states = 4 ** channels * p.keep
    step = 8 * states * states // 4
    keeps_steps = bool(p.algorithms) or p.fdm_flags
    return (3 + (nmax if keeps_steps else 0)) * step


class Server:
    def __init__(self, device: int = 0, hbm_budget: Optional[int] = None, max_active: int = 32):
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device: the server has no CPU fallback")
        self.device = device
        self.ctx = context(device)
        self.stream = torch.cuda.current_stream(torch.device("cuda", device))
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = int(0.5 * free)
        self.budget = hbm_budget
        self.max_active = max_active
        self.ticks = 0
        self.recalc_calls = 0  # merged recalculation calls (one per tick with terms)
        self.max_active_seen = 0
        self.blocks_per_tick: List[int] = []

    def serve(self, requests: List[Request], realtime: bool = True) -> List[Completed]:
        """Serve the stream; with realtime=False every request is taken as arrived at once."""
        pending = sorted(requests, key=lambda r: (r.arrival if realtime else 0.0, r.rid))
        active: List[list] = []  # [request, run, charged bytes, admitted time]
        out: List[Completed] = []
        t0 = time.perf_counter()

        def used() -> int:
            return sum(max(need, run.device_bytes()) for _, run, need, _ in active)
        while pending or active:
            now = time.perf_counter() - t0
            # admission: arrived, a free slot, and room in the budget (a run larger than the
            # whole budget is admitted alone)
            while pending and (not realtime or pending[0].arrival <= now) and len(active) < self.max_active:
                req = pending[0]
                params = RunParams.from_param(parse_param(req.param))
                data = read_data(req.data)
                need = run_bytes(params, data.nmax, data.channels)
                if active and used() + need > self.budget:
                    break
                pending.pop(0)
                run = QSRun(params, data, self.device, self.ctx)
                run.start()
                active.append([req, run, need, now])
            self.max_active_seen = max(self.max_active_seen, len(active))
            if not active:
                wait = pending[0].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.05))
                continue
            # one tick: every active run advances one NRG step
            jobs = [run.begin_step() for _, run, _, _ in active]
            ns, Hp, Ep, Vp = [], [], [], []
            for j in jobs:
                ns += j.ns
                Hp += j.Hp
                Ep += j.Ep
                Vp += j.Vp
            info = diag_batch_ptrs(ns, Hp, Ep, Vp, self.ctx, self.stream)
            self.ticks += 1
            self.blocks_per_tick.append(len(ns))
            terms: List[tuple] = []  # (GEMM3 terms, matrix sets they read)
            reads: List = []
            o = 0
            for (_, run, _, _), j in zip(active, jobs):
                run.deferred_terms, run.deferred_reads = terms, reads
                try:
                    run.end_step(j, info[o:o + len(j.ns)])
                finally:
                    run.deferred_terms = run.deferred_reads = None
                o += len(j.ns)
            if terms:
                gemm3_batch_array(np.concatenate([t for t, _ in terms]), self.ctx, self.stream)
                self.recalc_calls += 1
            del terms  # the operands they read may be reused from here on (stream-ordered)
            for gather in reads:
                gather()
            still = []
            for item in active:
                req, run, need, adm = item
                if run.done:
                    res = run.finish()
                    torch.cuda.synchronize(self.device)
                    out.append(Completed(req.rid, req.tag, res, req.arrival if realtime else 0.0, adm,
                                         time.perf_counter() - t0, run.nmax))
                else:
                    still.append(item)
            active = still
        return out


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times of a Poisson stream of n requests with the given mean rate (1/s)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def group_summary(done: List[Completed]) -> dict:
    """Latency of request groups -- the runs that share a tag, e.g. the twist values z of one
    z-averaged request -- from the group's arrival to the end of its last run."""
    groups: dict = {}
    for c in done:
        a, d = groups.get(c.tag, (c.arrival, c.done))
        groups[c.tag] = (min(a, c.arrival), max(d, c.done))
    lat = np.array([d - a for a, d in groups.values()])
    return {"groups": len(groups), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean())}


def summary(done: List[Completed], wall: float) -> dict:
    lat = np.array([c.latency for c in done])
    steps = sum(c.steps for c in done)
    return {"requests": len(done), "steps": steps, "wall_s": wall, "steps_per_s": steps / wall,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean())}
