"""Autotuner of the batched eigensolver's launch parameters (nrg_tuning, include/nrg_b200.h).

The eigensolver sends each block of a step down one of four paths by its order: the
one-CTA shared-memory solver (n <= small_max_n), the one-CTA shared-memory tridiagonal
reduction (n <= mid_max_n), the cluster reduction in distributed shared memory
(n <= cluster_max_n, when the clusters fit the SMs at once) and the streaming reduction
from HBM, whose CTAs run one, two or three per SM (reduction_ctas_per_sm). Where the crossovers
lie depends on the device, so they are measured, not assumed: the reference's own
scheduler (c++/core.hpp:98-107, c++/subspaces.hpp:103-123) only orders the blocks largest
first; on a GPU the choice of path per block is the equivalent decision.

Workloads (seeded, synthetic; the size mixes of the NRG steps this library serves; blocks
are diag(2^{-k/2}) plus symmetric N(0, 0.1^2) couplings, as in the benchmark):
  step   8 batches of 40 blocks, orders log-uniform in [8, 480] (the steps of an Anderson-model
         run at keep 1000)
  wide   2 batches of 300 blocks, orders log-uniform in [8, 1024] (many runs served at once)
  large  12 blocks in [800, 2000], 4 blocks in [1500, 4096] and 24 blocks in [200, 7049]
         (the steps of the keep-4000 Anderson and keep-5000 two-channel Kondo runs, bound by
         their largest blocks)
  bulk   1500 blocks in [8, 2048] (a seventh of the benchmark's batched-eigensolve step)
Each candidate is timed with CUDA events around nrg_diag_batch (the consumed inputs are
refreshed outside the timed region), best of `reps`; the objective is the mean over the
batches of the time relative to the starting parameters. Coordinate descent over the
parameters, each from the current best, twice round; a change is kept when it wins by more
than 2% (the batches of small blocks take a few milliseconds and vary by about that much).

The result is written to tuning.json beside this module, keyed by the device name, and
applied by nrgljubljana_b200.context() to every context it creates on such a device.
Run: python -m nrgljubljana_b200.autotune [--reps R]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")
SEED = 20261203

GRID = {
    "small_max_n": [32, 48, 64, 80, 96],
    "mid_max_n": [128, 160, 192, 224, 236],
    "cluster_max_n": [400, 480, 560, 600, 640],
    # The two-stage path's bulge chasing has a critical path of about 3n dependent steps; below
    # order ~2000 it is as long as the block's one-stage reduction, so lower thresholds only
    # pay where the other blocks of a batch hide it, and cost 10-15% on keep-4000 Anderson
    # steps (blocks up to 1622), measured.
    "band_min_n": [0, 2048, 3072, 4096],
    "reduction_ctas_per_sm": [1, 2, 3],
    "band_max_blocks": [4, 8, 16, 32, 64],
}
KEYS = ("small_max_n", "mid_max_n", "cluster_max_n", "reduction_ctas_per_sm", "band_min_n", "band_max_blocks")
# (batches, blocks per batch, smallest and largest order) of the timed workloads
WORKLOADS = ((8, 40, 8, 480), (2, 300, 8, 1024), (1, 12, 800, 2000), (1, 4, 1500, 4096), (1, 24, 200, 7049),
             (1, 1500, 8, 2048))


def device_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def load_table(device: int = 0) -> Optional[Dict[str, int]]:
    """The tuned parameters for this device's model from tuning.json, or None."""
    try:
        with open(TABLE) as f:
            tab = json.load(f)
    except (OSError, ValueError):
        return None
    try:
        name = device_name(device)
    except Exception:
        return None
    entry = tab.get(name)
    return dict(entry["tuning"]) if entry else None


def workloads() -> List[np.ndarray]:
    rng = np.random.Generator(np.random.PCG64(SEED))
    out = []
    for k, nb, nmin, nmax in WORKLOADS:
        for _ in range(k):
            u = rng.uniform(math.log(nmin), math.log(nmax), nb)
            out.append(np.clip(np.rint(np.exp(u)), nmin, nmax).astype(np.int64))
    return out


class _Batch:
    def __init__(self, torch, ctx, sizes: np.ndarray, dev, seed: int):
        import ctypes as C
        self.torch, self.ctx, self.sizes = torch, ctx, sizes
        offs = np.zeros(len(sizes) + 1, dtype=np.int64)
        offs[1:] = np.cumsum(sizes ** 2)
        voffs = np.zeros(len(sizes) + 1, dtype=np.int64)
        voffs[1:] = np.cumsum(sizes)
        self.pristine = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
        g = torch.Generator(device=dev)
        for b, n in enumerate(sizes.tolist()):
            g.manual_seed(seed * 1009 + b)
            h = torch.randn((n, n), generator=g, dtype=torch.float64, device=dev).mul_(0.1).triu_(1)
            h.diagonal().copy_(torch.pow(2.0, -torch.arange(n, dtype=torch.float64, device=dev) / 2.0))
            self.pristine[offs[b]:offs[b + 1]].view(n, n).copy_(h)
        self.work = torch.empty_like(self.pristine)
        self.evecs = torch.empty_like(self.pristine)
        self.evals = torch.empty(int(voffs[-1]), dtype=torch.float64, device=dev)
        nb = len(sizes)
        self.args = ((C.c_int * nb)(*sizes.tolist()),
                     (C.c_void_p * nb)(*[self.work.data_ptr() + 8 * int(o) for o in offs[:-1]]),
                     (C.c_void_p * nb)(*[self.evals.data_ptr() + 8 * int(o) for o in voffs[:-1]]),
                     (C.c_void_p * nb)(*[self.evecs.data_ptr() + 8 * int(o) for o in offs[:-1]]),
                     (C.c_int * nb)())
        self.offs, self.voffs = offs, voffs

    def time_once(self) -> float:
        torch = self.torch
        self.work.copy_(self.pristine)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n, H, E, V, info = self.args
        e0.record()
        rc = self.ctx.lib.nrg_diag_batch(self.ctx.ptr, len(self.sizes), n, H, E, V, info, None)
        e1.record()
        e1.synchronize()
        if rc != 0:
            from ._lib import last_error
            raise RuntimeError(f"nrg_diag_batch returned {rc}: {last_error()}")
        return e0.elapsed_time(e1)

    def max_residual(self) -> float:
        torch = self.torch
        worst = 0.0
        for b, n in enumerate(self.sizes.tolist()):
            h = self.pristine[self.offs[b]:self.offs[b + 1]].view(n, n)
            H = torch.triu(h) + torch.triu(h, 1).T
            v = self.evecs[self.offs[b]:self.offs[b + 1]].view(n, n)
            w = self.evals[self.voffs[b]:self.voffs[b + 1]]
            r = torch.linalg.norm(v @ H - w[:, None] * v, dim=1).max() / max(float(w.abs().max()), 1e-300)
            worst = max(worst, float(r))
        return worst


def tune(device: int = 0, reps: int = 3, verbose: bool = True) -> dict:
    import torch

    from .api import Context
    torch.cuda.set_device(device)
    ctx = Context(device)  # a fresh context: the table in force does not bias the sweep
    dev = torch.device("cuda", device)
    batches = [_Batch(torch, ctx, s, dev, i) for i, s in enumerate(workloads())]
    grid = dict(GRID)

    base: List[float] = []

    def timed(t: dict) -> List[float]:
        ctx.set_tuning(**t)
        out = []
        for b in batches:
            b.time_once()  # warm-up: workspace growth, first launch of a kernel
            out.append(min(b.time_once() for _ in range(reps)))
        return out

    def objective(ms: List[float]) -> float:
        """Mean time relative to the starting parameters, so that every workload counts alike."""
        return float(np.mean([m / b0 for m, b0 in zip(ms, base)]))

    best = ctx.tuning
    base = timed(best)
    best_obj = objective(base)
    sweep = [{"tuning": dict(best), "ms": base, "objective": best_obj}]
    t0 = time.perf_counter()
    for _ in range(2):
        changed = False
        for key in KEYS:
            for v in grid[key]:
                cand = dict(best, **{key: v})
                if cand == best or not (32 <= cand["small_max_n"] <= cand["mid_max_n"] <= cand["cluster_max_n"]):
                    continue
                if key == "band_max_blocks" and cand["band_min_n"] == 0:
                    continue
                ms = timed(cand)
                obj = objective(ms)
                sweep.append({"tuning": cand, "ms": ms, "objective": obj})
                if verbose:
                    print(f"  {cand} {obj:.4f} {[round(x, 2) for x in ms]}", flush=True)
                if obj < best_obj * 0.98:  # a change must win by more than the timing noise
                    best, best_obj, changed = cand, obj, True
        if not changed:
            break
    ctx.set_tuning(**best)
    for b in batches:  # the chosen parameters give correct eigenpairs on every batch
        b.time_once()
        r = b.max_residual()
        if not r <= 1e-12:
            raise RuntimeError(f"residual {r} with {best}")
    final = timed(best)
    return {"tuning": best, "objective": best_obj, "default_ms": base, "tuned_ms": final,
            "speedup_vs_default": float(np.mean([a / b for a, b in zip(base, final)])),
            "workloads": "; ".join(f"{k} x {nb} blocks log-uniform in [{lo}, {hi}]" for k, nb, lo, hi in WORKLOADS)
                         + " (seed 20261203), best of %d per batch; objective: mean time relative to the defaults" % reps,
            "sweep_s": time.perf_counter() - t0, "evaluations": len(sweep), "sweep": sweep}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--dry-run", action="store_true", help="print the result, do not write the table")
    a = ap.parse_args(argv)
    res = tune(a.device, a.reps)
    name = device_name(a.device)
    print(json.dumps({name: {k: v for k, v in res.items() if k != "sweep"}}, indent=1))
    if not a.dry_run:
        try:
            with open(a.out) as f:
                tab = json.load(f)
        except (OSError, ValueError):
            tab = {}
        tab[name] = res
        with open(a.out, "w") as f:
            json.dump(tab, f, indent=1)
            f.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
