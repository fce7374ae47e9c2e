"""Benchmark of the B200 NRG step core on the synthetic batched-eigensolve workload.

Workload (one "step"): 10,000 real symmetric FP64 blocks with orders drawn log-uniform in
[8, 2048] (numpy PCG64, seed 20261203); block b is diag(2^{-k/2}, k = 0..n-1) plus
symmetric Gaussian couplings N(0, 0.1^2) (torch CUDA generator seeded 20261203 * 100003
+ b), the shape of an NRG step's symmetry blocks. All blocks are diagonalised in one
batched call (nrg_diag_batch). Metric: FP64 eigensolve GFLOP/s counted as
F_eig(n) = (10/3) n^3 per block (tridiagonal reduction 4/3 n^3 + back-transform 2 n^3).

Arms:
  default           the library, inputs resident in HBM (a device-to-device refresh of the
                    consumed inputs is inside each timed step); e2e through the host-pointer
                    entry point nrg_diag_batch_host from pinned host memory.
  --impl reference  the reference's CPU path (the oracle restatement of diagonalise() with
                    LAPACK dsyev, OpenMP over blocks as diagonalisations_OpenMP) on all host
                    cores, on a stratified sample of the same blocks.
Multi-GPU (--gpus N under torchrun): independent replicas, one batch per GPU, no collective
on the data path; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20261203
NMIN, NMAX = 8, 2048
METRIC = "fp64_eig_gflops"
UNIT = "GFLOP/s"
WORKLOAD = ("synthetic batched eigensolve: {nblk} real symmetric FP64 blocks, n log-uniform in [{nmin}, {nmax}] "
            "(PCG64 seed 20261203), H = diag(2^-k/2) + symmetric N(0, 0.1^2) couplings")


def block_sizes(nblk: int, nmin: int = NMIN, nmax: int = NMAX) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(SEED))
    u = rng.uniform(math.log(nmin), math.log(nmax), nblk)
    return np.clip(np.rint(np.exp(u)), nmin, nmax).astype(np.int64)


def f_eig(n) -> float:
    n = np.asarray(n, dtype=np.float64)
    return float(np.sum(10.0 / 3.0 * n ** 3))


def tridiag_bytes(n: int, nb: int = 16) -> float:
    """Algorithmic HBM bytes of the one-stage blocked reduction of an n x n block: each column's
    symmetric matrix-vector product reads the trailing lower triangle once, and each panel of nb
    columns reads and writes the trailing lower triangle once in its rank-2nb update."""
    m = np.arange(1, n - 1, dtype=np.float64)  # trailing orders n-k-1 for k = 0..n-3
    symv = 8.0 * np.sum(m * (m + 1) / 2)
    pe = np.minimum(np.arange(nb, n - 2 + nb, nb), n - 2).astype(np.float64)
    t = n - pe
    upd = 16.0 * np.sum(t * (t + 1) / 2)
    return symv + upd


def make_block(torch, b: int, n: int, device):
    g = torch.Generator(device=device)
    g.manual_seed(SEED * 100003 + b)
    h = torch.randn((n, n), generator=g, dtype=torch.float64, device=device).mul_(0.1).triu_(1)
    h.diagonal().copy_(torch.pow(2.0, -torch.arange(n, dtype=torch.float64, device=device) / 2.0))
    return h


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.p, self.lines = gpu, None, []

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        busy = [x for x in sm if mx and x > 0.5 * mx] or sm
        return {"sm_mhz": float(np.median(busy)) if busy else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except OSError:
        return {}


def cpu_sample(sizes: np.ndarray, target_s: float, threads: int):
    """Stratified sample (every s-th block in size order) whose dsyev time on `threads`
    cores is about target_s, calibrated with a short dsyev timing."""
    from oracle import oracle
    rng = np.random.default_rng(0)
    cal = [np.triu(rng.standard_normal((384, 384))) for _ in range(max(1, threads))]
    oracle.blas_threads(1)
    t0 = time.perf_counter()
    oracle.diag_batch(cal, nthreads=threads)
    dt = time.perf_counter() - t0
    per_n3 = dt * threads / (len(cal) * 384.0 ** 3)  # core-seconds per n^3
    total = per_n3 * float(np.sum(sizes.astype(np.float64) ** 3)) / threads
    stride = max(1, int(math.ceil(total / target_s)))
    order = np.argsort(sizes, kind="stable")
    return order[stride // 2::stride], stride


def run_cpu(blocks, threads: int):
    from oracle import oracle
    oracle.blas_threads(1)
    n = np.array([b.shape[0] for b in blocks], dtype=np.int32)
    moff = np.zeros(len(n), dtype=np.int64)
    voff = np.zeros(len(n), dtype=np.int64)
    moff[1:] = np.cumsum(n.astype(np.int64) ** 2)[:-1]
    voff[1:] = np.cumsum(n.astype(np.int64))[:-1]
    H0 = np.concatenate([b.ravel() for b in blocks])
    V = np.zeros(int(n.sum()))
    Z = np.zeros_like(H0)
    H = H0.copy()
    t0 = time.perf_counter()
    bad = oracle.diag_batch_packed(n, moff, voff, H, V, Z, threads)
    dt = time.perf_counter() - t0
    if bad:
        raise RuntimeError(f"{bad} blocks failed in dsyev")
    return dt


def sample_blocks_host(torch, sizes, idx, device):
    out = []
    for b in idx:
        out.append(make_block(torch, int(b), int(sizes[b]), device).cpu().numpy())
    return out


def workload_config(sizes: np.ndarray, args, world: int) -> dict:
    """The `config` object of both arms (the same keys and values for the same workload)."""
    return {"workload": WORKLOAD.format(nblk=len(sizes), nmin=args.nmin, nmax=args.nmax), "nblk": int(len(sizes)),
            "sum_n3": float(np.sum(sizes.astype(float) ** 3)), "flop_per_step": f_eig(sizes),
            "input_bytes": int(8 * np.sum(sizes.astype(np.int64) ** 2)),
            "l2": "inputs larger than L2 (30 GB vs 126 MB)", "parallelism": f"replicas x{world}"}


def max_over_ranks(dist, x: float, device) -> float:
    """The largest x of all ranks; x itself without a process group. Every rank takes this
    collective step, also after its own failure (pass math.inf there), so that no rank is left
    waiting for another."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reference_arm(args, rank: int) -> None:
    import torch
    if rank != 0:
        return
    sizes = block_sizes(args.nblk, args.nmin, args.nmax)
    threads = os.cpu_count() or 1
    idx, stride = cpu_sample(sizes, args.cpu_seconds, threads)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    blocks = sample_blocks_host(torch, sizes, idx, dev)
    flop = f_eig(sizes[idx])
    for _ in range(args.warmup):
        run_cpu(blocks, threads)
    times = [run_cpu(blocks, threads) for _ in range(args.steps)]
    t = float(np.mean(times))
    value = flop / t / 1e9
    sample = (f"{len(idx)} of {args.nblk} blocks (every {stride}th in size order, sum n^3 = "
              f"{float(np.sum(sizes[idx].astype(float) ** 3)):.3e}); LAPACK dsyev, OpenMP over blocks, 1 BLAS thread each")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(sizes, args, args.gpus), "sample": sample,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nblk", type=int, default=10000)
    ap.add_argument("--nmin", type=int, default=NMIN, help="smallest block order (profiling cases)")
    ap.add_argument("--nmax", type=int, default=NMAX, help="largest block order (profiling cases)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64-peak", action="store_true", help="skip the cuBLAS DGEMM peak measurement")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-nrg", action="store_true", help="skip the whole-run NRG measurement")
    ap.add_argument("--no-per-block", action="store_true", help="skip the one-block-per-launch GPU comparator")
    ap.add_argument("--c2", action="store_true",
                    help="also run the keep-4000 Anderson DM-NRG workload (Nmax=60)")
    ap.add_argument("--c4", action="store_true", help="also serve the generated z-averaged request stream")
    ap.add_argument("--c4-requests", type=int, default=6, help="requests of the --c4 stream")
    ap.add_argument("--c3", action="store_true",
                    help="also run the two-channel Kondo FDM workload (keep=5000, Nmax=50; minutes)")
    ap.add_argument("--write-c0", default=None, metavar="DIR",
                    help="write the param and data files of the NRG-run workload to DIR and exit")
    ap.add_argument("--write-c3", default=None, metavar="DIR",
                    help="write the param and data files of the two-channel Kondo FDM workload to DIR and exit")
    ap.add_argument("--c3-keep", type=int, default=5000, help="keep of --write-c3 (smaller cases for profiling)")
    ap.add_argument("--c3-nmax", type=int, default=50, help="Nmax of --write-c3")
    args = ap.parse_args()
    for out_dir, make in ((args.write_c0, c0_inputs), (args.write_c3, lambda: c3_inputs(args.c3_keep, args.c3_nmax))):
        if out_dir:
            os.makedirs(out_dir, exist_ok=True)
            param, data = make()
            for name, text in (("param", param), ("data", data)):
                with open(os.path.join(out_dir, name), "w") as f:
                    f.write(text)
    if args.write_c0 or args.write_c3:
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import nrgljubljana_b200 as nb
    ctx = nb.context(local)

    sizes = block_sizes(args.nblk, args.nmin, args.nmax)
    offs = np.zeros(args.nblk + 1, dtype=np.int64)
    offs[1:] = np.cumsum(sizes.astype(np.int64) ** 2)
    voffs = np.zeros(args.nblk + 1, dtype=np.int64)
    voffs[1:] = np.cumsum(sizes)
    total = int(offs[-1])
    dev = torch.device("cuda", local)
    pristine = torch.empty(total, dtype=torch.float64, device=dev)
    for b in range(args.nblk):
        n = int(sizes[b])
        pristine[offs[b]:offs[b + 1]].view(n, n).copy_(make_block(torch, b, n, dev))
    work = torch.empty_like(pristine)
    evecs = torch.empty_like(pristine)
    evals = torch.empty(int(voffs[-1]), dtype=torch.float64, device=dev)
    import ctypes as C
    nbk = args.nblk
    n_c = (C.c_int * nbk)(*[int(x) for x in sizes])
    Hp = (C.c_void_p * nbk)(*[work.data_ptr() + 8 * int(offs[b]) for b in range(nbk)])
    Vp = (C.c_void_p * nbk)(*[evecs.data_ptr() + 8 * int(offs[b]) for b in range(nbk)])
    Ep = (C.c_void_p * nbk)(*[evals.data_ptr() + 8 * int(voffs[b]) for b in range(nbk)])
    info = (C.c_int * nbk)()

    def step():
        work.copy_(pristine)
        rc = ctx.lib.nrg_diag_batch(ctx.ptr, nbk, n_c, Hp, Ep, Vp, info, None)
        if rc != 0:
            raise RuntimeError(f"nrg_diag_batch returned {rc}: {nb.load_library().nrg_last_error().decode()}")

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ctx.profile(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    elapsed = e0.elapsed_time(e1) / 1e3
    phases = ctx.profile_read()
    ctx.profile(False)
    elapsed = max_over_ranks(dist, elapsed, dev)
    flop_step = f_eig(sizes)
    value = world * args.steps * flop_step / elapsed / 1e9
    launches = int(sum(v[1] for v in phases.values()))

    # roofline of the dominant kernel
    peaks = measured_peaks()
    top = max(phases.items(), key=lambda kv: kv[1][0])
    roof = None
    # DRAM bytes per launch of tridiag_kernel relative to its algorithmic bytes, from one ncu
    # capture of the kernel as the benchmark's batch launches it (three CTAs per SM, the slabs
    # of the trailing triangle loaded with an L2 evict-first hint, the panel vectors with an
    # evict-last one) on 1400 blocks of n = 608: dram__bytes_read.sum + dram__bytes_write.sum =
    # 516.49 + 28.50 GB for 467.99 GB algorithmic; the ratio carries over to larger launches
    # because both grow with the per-column reads of the trailing triangle.
    tridiag_traffic_ratio = (516.49 + 28.50) / 467.99
    if top[0] == "tridiag":
        per_launch_bytes = args.steps * sum(tridiag_bytes(int(n)) for n in sizes if n > 64) / top[1][1]
        avg = top[1][0] / 1e3 / top[1][1]
        ach = per_launch_bytes / avg / 1e9
        pk = peaks.get("hbm_gbs", 6650.0)
        roof = {"kernel": "tridiag_kernel", "bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s",
                "frac": ach / pk, "traffic": per_launch_bytes * tridiag_traffic_ratio,
                "traffic_source": "ncu dram bytes of tridiag_kernel (three CTAs per SM) on 1400 x n=608 (profiles/tridiag_kernel_1400x608.md), scaled by algorithmic bytes",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "bytes_per_launch": per_launch_bytes, "avg_launch_ms": avg * 1e3}
    else:
        roof = {"kernel": top[0], "bound": "tensor", "achieved": None, "peak": None, "unit": "TFLOP/s",
                "frac": None, "traffic": None}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(sizes, args, world),
            "timing": "inputs resident in HBM; the consumed inputs are refreshed by a D2D copy inside each step",
            "steps_per_s": world * args.steps / elapsed, "gpu_launches": launches, "roofline": roof,
            "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items()},
            "clocks": clk.summary()}

    # validation: residuals and orthogonality of a sample of the last step's blocks (all 20
    # largest and 150 more, seeded), computed from the pristine inputs on the device
    try:
        vrng = np.random.default_rng(SEED)
        pick = sorted(set(vrng.choice(nbk, min(150, nbk), replace=False).tolist())
                      | set(np.argsort(sizes)[-20:].tolist()))
        worst_r = worst_o = 0.0
        for b in pick:
            n = int(sizes[b])
            h = pristine[offs[b]:offs[b + 1]].view(n, n)
            Hf = torch.triu(h) + torch.triu(h, 1).T
            v = evecs[offs[b]:offs[b + 1]].view(n, n)
            w = evals[voffs[b]:voffs[b + 1]]
            nrm = max(float(w.abs().max()), 1e-300)
            worst_r = max(worst_r, float(torch.linalg.norm(v @ Hf - w[:, None] * v, dim=1).max()) / nrm)
            worst_o = max(worst_o, float((v @ v.T - torch.eye(n, dtype=torch.float64, device=dev)).abs().max()))
        line["validation"] = {"blocks": len(pick), "max_residual_rel": worst_r, "max_orthogonality_err": worst_o,
                              "ok": worst_r <= 1e-10 and worst_o <= 1e-9}
    except (RuntimeError, MemoryError) as err:
        line["validation"] = {"error": str(err)[:200]}
    del work, evecs, evals
    torch.cuda.empty_cache()
    if not args.no_cpu and rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        idx, stride = cpu_sample(sizes, args.cpu_seconds, threads)
        blocks = [pristine[offs[b]:offs[b + 1]].view(int(sizes[b]), int(sizes[b])).cpu().numpy() for b in idx]
        t = run_cpu(blocks, threads)
        cpu_v = f_eig(sizes[idx]) / t / 1e9
        line["cpu_baseline"] = {"value": cpu_v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{len(idx)} of {nbk} blocks (every {stride}th in size order), {t:.1f} s"}
    if not args.no_per_block and rank == 0 and world == 1:
        line["per_block_gpu"] = per_block_arm(torch, pristine, sizes, offs, dev)
    if rank == 0 and not args.no_fp64_peak:
        line["fp64_peak"] = fp64_peak(torch, dev)
        pk = line["fp64_peak"].get("burst_tflops")
        if pk:
            line["fp64_frac"] = {"achieved_tflops": value / world / 1e3, "peak_tflops": pk,
                                 "frac": value / world / 1e3 / pk,
                                 "peak_source": "cuBLAS DGEMM 8192^3 measured in this run, best of 10"}
    if not args.no_e2e:  # every rank: its own replica through the host API, max over ranks
        # The device-resident inputs go to pinned host memory; the device copy and the context's
        # workspace are given back, so the host path runs within its own bounded ring.
        hostH = torch.empty(pristine.numel(), dtype=torch.float64, pin_memory=True)
        hostH.copy_(pristine)
        del pristine
        torch.cuda.empty_cache()
        ctx.trim()
        e2e = e2e_arm(torch, ctx, hostH, sizes, offs, voffs, args, dist, dev)
        del hostH
        if rank == 0:
            line["e2e"] = e2e
    else:
        del pristine
    torch.cuda.empty_cache()
    if not args.no_nrg and rank == 0:
        line["nrg_run"] = nrg_run_arm(torch, local, args)
    if not args.no_nrg and rank == 0:
        line["serving"] = serving_arm(torch, local, line["nrg_run"])
    if args.c2 and rank == 0:
        torch.cuda.empty_cache()
        try:
            line["c2_run"] = c2_arm(torch, local, args)
        except (RuntimeError, MemoryError) as err:
            line["c2_run"] = {"workload": C2_WORKLOAD, "error": str(err)[:300]}
    if args.c4 and rank == 0:
        torch.cuda.empty_cache()
        try:
            line["c4_serving"] = c4_arm(torch, local, args)
        except (RuntimeError, MemoryError) as err:
            line["c4_serving"] = {"workload": C4_WORKLOAD, "error": str(err)[:300]}
    if args.c3 and rank == 0:
        torch.cuda.empty_cache()
        try:
            line["c3_run"] = c3_arm(torch, local, args)
        except (RuntimeError, MemoryError) as err:
            line["c3_run"] = {"workload": C3_WORKLOAD, "error": str(err)[:600]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def fp64_peak(torch, dev, n: int = 8192, reps: int = 10, sustain_s: float = 4.0) -> dict:
    """The FP64 denominator of the eigensolver's roofline: a cuBLAS DGEMM of n x n x n
    (torch.matmul on float64), best of `reps` timed singly with CUDA events (burst), and the
    mean over a loop of about `sustain_s` seconds (sustained), with the SM clocks sampled
    during the loop."""
    a = torch.randn((n, n), dtype=torch.float64, device=dev)
    b = torch.randn((n, n), dtype=torch.float64, device=dev)
    c = torch.empty_like(a)
    flop = 2.0 * n ** 3
    for _ in range(3):
        torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = math.inf
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    k = max(1, int(sustain_s / best))
    with ClockSampler(dev.index or 0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
    mean = e0.elapsed_time(e1) / 1e3 / k
    del a, b, c
    torch.cuda.empty_cache()
    return {"gemm": f"cuBLAS DGEMM {n}^3 (torch.matmul, float64)", "burst_tflops": flop / best / 1e12,
            "sustained_tflops": flop / mean / 1e12, "sustained_loop": k, "clocks": clk.summary()}


def per_block_arm(torch, pristine, sizes, offs, dev, target_flop: float = 1.5e12) -> dict:
    """The plain GPU path: one cuSOLVER eigensolve (torch.linalg.eigh) per block and launch,
    on a size-stratified sample of the same blocks; GFLOP/s on the same F_eig count."""
    order = np.argsort(sizes, kind="stable")
    f = np.array([f_eig(int(n)) for n in sizes[order]])
    stride = max(1, int(math.ceil(f.sum() / target_flop)))
    idx = order[::stride]
    mats = [pristine[offs[b]:offs[b + 1]].view(int(sizes[b]), int(sizes[b])) for b in idx]
    for h in mats[:8]:
        torch.linalg.eigh(h, UPLO="U")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for h in mats:
        w, q = torch.linalg.eigh(h, UPLO="U")
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    return {"value": f_eig(sizes[idx]) / t / 1e9, "unit": UNIT, "impl": "torch.linalg.eigh (cuSOLVER) per block",
            "sample": f"{len(idx)} of {len(sizes)} blocks (every {stride}th in size order)", "seconds": t}


C0_PARAM = """[param]
symtype=QS
model=SIAM
U=1.0
Gamma=0.04
delta=0
band=flat
discretization=Z
Lambda=2
z=1
keep=1000
keepenergy=10
T=1e-8
ops=n_d A_d
dmnrg=true
specd=A_d-A_d
"""
C0_SPEC = "spec_DMNRG_dens_A_d-A_d"  # the DM-NRG spectral function of the C0 run

NRG_WORKLOAD = ("NRG run, QS single-impurity Anderson model U=1, eps_d=-0.5 (delta=0), Gamma=0.04, flat band, "
                "Lambda=2 (Z), z=1, Nmax=40, keep=1000, keepenergy=10, T=1e-8, operator n_d, DM-NRG spectral "
                "function A_d-A_d (1000 bins/decade, broadened); input generated by nrgljubljana_b200.datagen")


C3_PARAM = """[param]
symtype=QS
Lambda=3
keep=5000
T=1e-6
fdm=true
spect=S_imp-S_imp
"""
C3_WORKLOAD = ("NRG run, QS two-channel Kondo model, impurity spin 1/2, J=0.2 on both flat channels, "
               "Lambda=3 (Z), z=1, Nmax=50, keep=5000, T=1e-6, FDM dynamic spin susceptibility S_imp-S_imp "
               "(1000 bins/decade, broadened) and FDM thermodynamics; input generated by nrgljubljana_b200.datagen")


C2_PARAM = """[param]
symtype=QS
model=SIAM
U=1.0
Gamma=0.04
delta=0
band=flat
discretization=Z
Lambda=2
z=1
keep=4000
T=1e-8
ops=n_d A_d
dmnrg=true
specd=A_d-A_d
bins=10
emin=1e-10
emax=1
"""
C2_WORKLOAD = ("NRG run, QS single-impurity Anderson model U=1, eps_d=-0.5 (delta=0), Gamma=0.04, flat band, "
               "Lambda=2 (Z), z=1, Nmax=60, keep=4000, T=1e-8, operators n_d and A_d, DM-NRG spectral function "
               "A_d-A_d in 10 bins per decade over [1e-10, 1] (101 bins per sign), broadened; input generated by "
               "nrgljubljana_b200.datagen")


def per_block_driver(torch):
    """The same NRG-run driver with the plain GPU eigensolver: one cuSOLVER eigh
    (torch.linalg.eigh) per block and launch, in place of the batched nrg_diag_batch."""
    from nrgljubljana_b200.nrg_run import QSRun

    class PerBlock(QSRun):
        def _diagonalise(self, job):
            for b, n in enumerate(job.ns):
                h = job.Hbuf[job.moff[b]:job.moff[b + 1]].view(n, n)
                w, q = torch.linalg.eigh(h, UPLO="U")
                job.Ebuf[job.voff[b]:job.voff[b + 1]].copy_(w)
                job.Vbuf[job.moff[b]:job.moff[b + 1]].view(n, n).copy_(q.T)
            return np.zeros(len(job.ns), dtype=np.int32)
    return PerBlock


def c2_inputs():
    from nrgljubljana_b200.datagen import siam_qs
    return C2_PARAM, siam_qs(1.0, 0.0, 0.04, 2.0, 60, 1.0, "Z", ops=["n_d", "A_d"])


def c2_arm(torch, device: int, args) -> dict:
    """One whole run of the keep-4000 Anderson DM-NRG workload (wall clock, device synchronised),
    beside the same driver with one cuSOLVER eigh per block and launch; the CPU dsyev path
    estimated as for the two-channel run."""
    from nrgljubljana_b200 import context
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import QSRun, RunParams
    param, data = c2_inputs()
    p, d = RunParams.from_param(parse_param(param)), read_data(data)
    ctx = context(device)

    PerBlock = per_block_driver(torch)

    def timed(cls):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = cls(p, d, device, ctx).run()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, res
    torch.cuda.reset_peak_memory_stats(device)
    t, res = timed(QSRun)
    peak = torch.cuda.max_memory_allocated(device) / 2 ** 30
    t_pb, res_pb = timed(PerBlock)
    flop = sum(f_eig(np.array(ns)) for ns in res.block_dims)
    td, tdp = np.array(res.td), np.array(res_pb.td)
    big = np.abs(td) >= 1e-6
    a = res.spectra["spec_DMNRG_dens_A_d-A_d"][:, 1]
    b = res_pb.spectra["spec_DMNRG_dens_A_d-A_d"][:, 1]
    out = {"workload": C2_WORKLOAD, "steps_per_run": d.nmax, "steps_per_s": d.nmax / t, "s_per_run": t,
           "timing": "wall clock of one run (host driver included)", "eig_flop_per_run": flop,
           "blocks_per_step_max": max(res.blocks_per_step), "block_dim_max": max(res.max_dim_per_step),
           "peak_device_gib": peak,
           "per_block_gpu": {"steps_per_s": d.nmax / t_pb, "s_per_run": t_pb,
                             "impl": "same driver, torch.linalg.eigh (cuSOLVER) one block per launch",
                             "td_max_rel_diff": float(np.max(np.abs(tdp[big] - td[big]) / np.abs(td[big]))),
                             "spectrum_max_diff_rel_to_peak": float(np.max(np.abs(a - b)) / np.max(np.abs(a)))}}
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        heavy = max(range(len(res.block_dims)), key=lambda k: sum(float(n) ** 3 for n in res.block_dims[k]))
        est = cpu_dsyev_estimate(res.block_dims[heavy], threads)
        c1 = est["measured"]["dsyev_1_thread_s"]["1200"] / 1200.0 ** 3
        tot_i = 0.0
        for ns in res.block_dims:
            load = np.zeros(threads)
            for n in sorted(ns, reverse=True):
                load[np.argmin(load)] += c1 * float(n) ** 3
            tot_i += float(load.max())
        scale = sum(sum(float(n) ** 3 for n in ns) for ns in res.block_dims) / \
            sum(float(n) ** 3 for n in res.block_dims[heavy])
        per_run = {"openmp_over_blocks_s": tot_i, "threaded_blas_s": est["threaded_blas_s"] * scale}
        out["cpu_baseline"] = {"steps_per_s_estimated": d.nmax / min(per_run.values()),
                               "diag_s_per_run_estimated": per_run, "cores": threads, "kind": "port",
                               "sample": "dsyev of n = 600, 1200 (1 thread) and 2000 (all threads), scaled by n^3 "
                                         "to every block of the run; diagonalisations only",
                               "measured": est["measured"]}
    return out


C4_WORKLOAD = ("serving: a Poisson stream (mean 4 requests/s, seed 20261203) of z-averaged QS Anderson-model "
               "requests, each eps_d ~ U[-0.7, -0.3] (delta = eps_d + 0.5), U = 1, Gamma ~ U[0.02, 0.08], "
               "keep ~ U{1000..3000}, Nmax = 50, Lambda = 2, and 8-32 twist values z ~ U(0, 1], one run per z; "
               "inputs generated by nrgljubljana_b200.datagen; runs admitted by slots (16) and HBM budget")


def _c4_data(args):
    from nrgljubljana_b200.datagen import siam_qs
    delta, gam, z = args
    return siam_qs(1.0, delta, gam, 2.0, 50, z, "Z", ops=["n_d"])


def c4_requests(nreq: int, seed: int = SEED):
    """The seeded requests of the serving workload: one Request per (request, z), tag = request.
    The inputs are generated on all host cores (a spawned process pool: the parent already
    holds a CUDA context)."""
    import multiprocessing
    from concurrent.futures import ProcessPoolExecutor
    from nrgljubljana_b200.serve import Request, poisson_arrivals
    rng = np.random.default_rng(seed)
    arr = poisson_arrivals(nreq, 4.0, seed)
    specs = []
    for k in range(nreq):
        eps = rng.uniform(-0.7, -0.3)
        gam = rng.uniform(0.02, 0.08)
        keep = int(rng.integers(1000, 3001))
        nz = int(rng.integers(8, 33))
        zs = 1.0 - rng.random(nz)  # (0, 1]
        for z in zs:
            specs.append((k, eps + 0.5, gam, keep, float(z)))
    with ProcessPoolExecutor(max_workers=os.cpu_count() or 1, mp_context=multiprocessing.get_context("spawn")) as ex:
        datas = list(ex.map(_c4_data, [(dl, g, z) for _, dl, g, _, z in specs], chunksize=1))
    out = []
    for rid, ((k, delta, gam, keep, z), data) in enumerate(zip(specs, datas)):
        param = (f"[param]\nsymtype=QS\nmodel=SIAM\nU=1.0\nGamma={gam!r}\ndelta={delta!r}\n"
                 f"band=flat\ndiscretization=Z\nLambda=2\nz={z!r}\nkeep={keep}\nT=1e-8\nops=n_d\n")
        out.append(Request(rid, param, data, float(arr[k]), f"request{k}"))
    return out


def c4_arm(torch, device: int, args) -> dict:
    """The serving workload with generated requests, served in real time; the first run is
    also run alone and its thermodynamics compared bit for bit with the one from the mix."""
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import QSRun, RunParams
    from nrgljubljana_b200.serve import Server, group_summary, summary
    t0 = time.perf_counter()
    reqs = c4_requests(args.c4_requests)
    t_gen = time.perf_counter() - t0
    srv = Server(device, max_active=16)
    t0 = time.perf_counter()
    done = srv.serve(reqs, realtime=True)
    wall = time.perf_counter() - t0
    out = {"workload": C4_WORKLOAD, "requests": args.c4_requests, "runs": len(reqs),
           "input_generation_s": t_gen, "runs_summary": summary(done, wall), "requests_summary": group_summary(done),
           "max_blocks_per_tick": max(srv.blocks_per_tick)}
    first = min(done, key=lambda c: c.rid)
    r0 = reqs[first.rid]
    alone = QSRun(RunParams.from_param(parse_param(r0.param)), read_data(r0.data), device).run()
    # Alone, a run's large blocks go to the cluster reduction; in a full tick to the one-CTA
    # reduction (the kernel choice depends on the batch): same arithmetic, another summation
    # order, so the results agree to round-off rather than bit for bit -- while the truncation
    # keeps the same states. A hard cut at `keep` inside a near-degeneracy can keep different
    # multiplets after round-off differences; the comparison covers the steps before that.
    k = next((j for j, (x, y) in enumerate(zip(alone.block_dims, first.result.block_dims)) if x != y),
             len(alone.block_dims))
    a, m = np.array(alone.td[:k + 1]), np.array(first.result.td[:k + 1])
    big = np.abs(a) >= 1e-6  # values that vanish by symmetry are round-off noise in every run
    out["alone_vs_mix"] = {"bitwise_equal": bool(np.array_equal(np.array(alone.td), np.array(first.result.td))),
                           "steps_with_same_kept_states": k, "steps": len(alone.block_dims),
                           "td_max_rel_diff_over_those_steps":
                               float(np.max(np.abs(a[big] - m[big]) / np.abs(a[big]))) if big.any() else 0.0,
                           "tolerance": 1e-10}
    return out


def c3_inputs(keep: int = 5000, nmax: int = 50):
    from nrgljubljana_b200.datagen import kondo_qs
    return C3_PARAM.replace("keep=5000", f"keep={keep}"), kondo_qs([0.2, 0.2], 0.5, 3.0, nmax, ops=["S_imp"])


def cpu_dsyev_estimate(dims, threads: int) -> dict:
    """The CPU time of one step's diagonalisations (dsyev, eigenvalues and vectors) on the host
    cores, estimated from measured sample blocks: t(n) = c n^3 fitted on single-thread dsyev
    of n = 600 and 1200 (layout i: OpenMP over blocks, one BLAS thread each, as
    diagonalisations_OpenMP runs; the step takes the longest-processing-time schedule of the
    blocks on `threads` cores) and on threaded dsyev of n = 2000 (layout ii: blocks one after
    another, all BLAS threads)."""
    from oracle import oracle as O
    rng = np.random.default_rng(SEED)

    def block(n):
        h = np.triu(rng.standard_normal((n, n)) * 0.1, 1)
        h[np.diag_indices(n)] = 2.0 ** (-np.arange(n) / 2.0)
        return h
    O.build()
    O.blas_threads(1)
    t1 = {}
    for n in (600, 1200):
        h = block(n)
        t0 = time.perf_counter()
        O.diagonalise(h)
        t1[n] = time.perf_counter() - t0
    c1 = t1[1200] / 1200.0 ** 3
    O.blas_threads(threads)
    h = block(2000)
    t0 = time.perf_counter()
    O.diagonalise(h)
    tt = time.perf_counter() - t0
    O.blas_threads(1)
    ct = tt / 2000.0 ** 3
    load = np.zeros(threads)
    for n in sorted(dims, reverse=True):  # longest processing time first
        load[np.argmin(load)] += c1 * float(n) ** 3
    return {"openmp_over_blocks_s": float(load.max()),
            "threaded_blas_s": float(sum(ct * float(n) ** 3 for n in dims)),
            "measured": {"dsyev_1_thread_s": {str(k): v for k, v in t1.items()},
                         f"dsyev_{threads}_threads_n2000_s": tt}}


def c3_arm(torch, device: int, args) -> dict:
    """One whole run of the two-channel Kondo FDM workload: the forward sweep (assembly, batched
    eigensolve, recalculation) and the FDM density matrices and spectral pass, wall clock on the
    device; the reference's CPU dsyev path on the host cores estimated for the same steps."""
    from nrgljubljana_b200 import context
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import QSRun, RunParams
    param, data = c3_inputs()
    p, d = RunParams.from_param(parse_param(param)), read_data(data)
    ctx = context(device)
    torch.cuda.reset_peak_memory_stats(device)
    run = QSRun(p, d, device, ctx)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    try:
        run.start()
        while not run.done:
            job = run.begin_step()
            run.end_step(job, run._diagonalise(job))
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        res = run.finish()
    except Exception as err:  # where the memory went, for the report
        free, total = torch.cuda.mem_get_info(device)
        raise RuntimeError(f"step {run.N}: {err}; device: {torch.cuda.memory_allocated(device) / 2 ** 30:.1f} GiB "
                           f"allocated, {torch.cuda.memory_reserved(device) / 2 ** 30:.1f} reserved by torch, "
                           f"{free / 2 ** 30:.1f} of {total / 2 ** 30:.1f} free; "
                           f"{run.spilled_bytes / 2 ** 30:.1f} GiB of eigenvectors in host memory") from err
    torch.cuda.synchronize()
    t_all = time.perf_counter() - t0
    flop = sum(f_eig(np.array(ns)) for ns in res.block_dims)
    out = {"workload": C3_WORKLOAD, "steps_per_run": d.nmax, "steps_per_s": d.nmax / t_all,
           "s_per_run": t_all, "forward_s": t_fwd, "fdm_and_spectra_s": t_all - t_fwd,
           "timing": "wall clock of one run (host driver included)",
           "eig_flop_per_run": flop, "eig_gflops_forward": flop / t_fwd / 1e9,
           "blocks_per_step_max": max(res.blocks_per_step), "block_dim_max": max(res.max_dim_per_step),
           "peak_device_gib": torch.cuda.max_memory_allocated(device) / 2 ** 30,
           "eigenvectors_stored_gib": sum(8.0 * sum(n * n for n in ns) for ns in res.block_dims) / 2 ** 30,
           "eigenvectors_via_host_gib": run.spilled_bytes / 2 ** 30,
           "tdfdm": dict(zip(*res.tdfdm)) if res.tdfdm else None,
           "spectrum": {k: int(len(v)) for k, v in res.spectra.items()}}
    if not args.no_per_block:
        # Parity and the plain GPU path: the same run with one cuSOLVER eigh per block and launch.
        # The comparison covers the steps whose kept states agree (a hard cut at keep inside a
        # near-degeneracy may keep another multiplet after a round-off difference).
        td, blk = np.array(res.td), res.block_dims
        del run, job
        torch.cuda.empty_cache()
        PerBlock = per_block_driver(torch)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res_pb = PerBlock(p, d, device, ctx).run()
        torch.cuda.synchronize()
        t_pb = time.perf_counter() - t0
        k = next((j for j, (x, y) in enumerate(zip(blk, res_pb.block_dims)) if sorted(x) != sorted(y)), len(blk))
        tdp = np.array(res_pb.td)
        big = np.abs(td[:k]) >= 1e-6
        name = next(iter(res.spectra))
        a, b = res.spectra[name][:, 1], res_pb.spectra[name][:, 1]
        out["per_block_gpu"] = {"steps_per_s": d.nmax / t_pb, "s_per_run": t_pb,
                                "impl": "same driver, torch.linalg.eigh (cuSOLVER) one block per launch"}
        out["parity"] = {"against": "the per-block cuSOLVER run of the same driver",
                         "steps_with_same_kept_states": k, "steps": len(blk),
                         "td_max_rel_diff": float(np.max(np.abs(tdp[:k][big] - td[:k][big]) / np.abs(td[:k][big]))),
                         "tdfdm_rel_diff": {f: float(abs(x - y) / max(abs(x), 1e-300))
                                            for f, x, y in zip(res.tdfdm[0], res.tdfdm[1], res_pb.tdfdm[1])},
                         "spectrum_max_diff_rel_to_peak": float(np.max(np.abs(a - b)) / np.max(np.abs(a)))
                         if a.shape == b.shape else None}
    if not args.no_cpu:
        threads = os.cpu_count() or 1
        heavy = max(range(len(res.block_dims)), key=lambda k: sum(float(n) ** 3 for n in res.block_dims[k]))
        est = cpu_dsyev_estimate(res.block_dims[heavy], threads)
        scale = sum(sum(float(n) ** 3 for n in ns) for ns in res.block_dims) / \
            sum(float(n) ** 3 for n in res.block_dims[heavy])
        # layout i: every step's own schedule of its blocks on the cores
        tot_i = 0.0
        c1 = est["measured"]["dsyev_1_thread_s"]["1200"] / 1200.0 ** 3
        for ns in res.block_dims:
            load = np.zeros(threads)
            for n in sorted(ns, reverse=True):
                load[np.argmin(load)] += c1 * float(n) ** 3
            tot_i += float(load.max())
        per_run = {"openmp_over_blocks_s": tot_i, "threaded_blas_s": est["threaded_blas_s"] * scale}
        best = min(per_run.values())
        out["cpu_baseline"] = {"steps_per_s_estimated": d.nmax / best, "diag_s_per_run_estimated": per_run,
                               "cores": threads, "kind": "port",
                               "sample": "dsyev of n = 600, 1200 (1 thread) and 2000 (all threads), scaled by n^3 "
                                         "to every block of the run; diagonalisations only (the reference's "
                                         "recalculation and FDM sums come on top)",
                               "measured": est["measured"]}
    return out


def c0_inputs():
    from nrgljubljana_b200.datagen import siam_qs
    return C0_PARAM, siam_qs(1.0, 0.0, 0.04, 2.0, 40, 1.0, "Z", ops=["n_d", "A_d"])


SERVE_MIX = ["legacy_Himp", "legacy_simple", "test12_Nmax", "test35_betabar", "test15_safeguard",
             "test13_strategy_all", "test0_minimal", "test200_data_has"]


def serving_arm(torch, device: int, single: dict) -> dict:
    """The serving loop: (1) saturation -- 16 runs of the reference's regression inputs
    submitted at once, one batched eigensolve per tick; (2) a Poisson stream of 32 requests
    at a mean 4 runs/s drawn from the same inputs (seed 20261203); steps/s and p50/p99
    latency from arrival to result."""
    from nrgljubljana_b200.serve import Request, Server, poisson_arrivals, summary
    base = os.path.join(ROOT, "tests", "golden", "nrg")
    texts = {c: (open(os.path.join(base, c, "param")).read(), open(os.path.join(base, c, "data")).read())
             for c in SERVE_MIX}
    mix = SERVE_MIX + SERVE_MIX
    reqs = [Request(i, *texts[c], 0.0, c) for i, c in enumerate(mix)]
    Server(device).serve(reqs[:4], realtime=False)  # warm-up
    torch.cuda.synchronize()
    srv = Server(device, max_active=16)
    t0 = time.perf_counter()
    done = srv.serve(reqs, realtime=False)
    sat = summary(done, time.perf_counter() - t0)
    sat["max_blocks_per_tick"] = max(srv.blocks_per_tick)
    rng = np.random.default_rng(SEED)
    arr = poisson_arrivals(32, 4.0, SEED)
    picks = [SERVE_MIX[k] for k in rng.integers(0, len(SERVE_MIX), size=32)]
    stream = [Request(i, *texts[c], float(arr[i]), c) for i, c in enumerate(picks)]
    srv = Server(device, max_active=16)
    t0 = time.perf_counter()
    done = srv.serve(stream, realtime=True)
    poi = summary(done, time.perf_counter() - t0)
    # the plain GPU path on the same 16-run mix: the same driver with one cuSOLVER eigh per block
    # and launch, runs one after another
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import RunParams
    PerBlock = per_block_driver(torch)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps = 0
    for r in reqs:
        res = PerBlock(RunParams.from_param(parse_param(r.param)), read_data(r.data), device).run()
        steps += len(res.block_dims)
    torch.cuda.synchronize()
    t_pb = time.perf_counter() - t0
    pb = {"steps_per_s": steps / t_pb, "wall_s": t_pb, "steps": steps,
          "impl": "same driver, torch.linalg.eigh (cuSOLVER) one block per launch, the 16 runs one after another"}
    return {"workload": "runs of the reference's regression inputs " + ", ".join(SERVE_MIX),
            "saturation_16_runs": sat, "poisson_4_per_s_32_requests": poi,
            "single_run_steps_per_s": single["steps_per_s"], "per_block_gpu_same_mix": pb,
            "served_over_per_block": sat["steps_per_s"] / pb["steps_per_s"]}


def nrg_run_arm(torch, device: int, args) -> dict:
    """Whole NRG runs (host driver + device step core) in NRG steps/s, beside the same run
    with one cuSOLVER call per block and the CPU restatement on all host cores."""
    from nrgljubljana_b200 import context
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import QSRun, RunParams
    param, data = c0_inputs()
    p, d = RunParams.from_param(parse_param(param)), read_data(data)
    ctx = context(device)

    PerBlock = per_block_driver(torch)

    spilled = []

    def timed(cls, reps):
        cls(p, d, device).run()  # warm-up
        torch.cuda.synchronize()
        best, res = None, None
        for _ in range(reps):
            t0 = time.perf_counter()
            run = cls(p, d, device)
            res = run.run()
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
            spilled.append(run.spilled_bytes)
        return best, res

    ctx.profile(True)
    ctx.profile_read()
    t_b200, res = timed(QSRun, 3)
    phases = ctx.profile_read()
    ctx.profile(False)
    t_pb, res_pb = timed(PerBlock, 1)
    out = {"workload": NRG_WORKLOAD, "steps_per_run": d.nmax, "steps_per_s": d.nmax / t_b200,
           "ms_per_run": t_b200 * 1e3, "timing": "wall clock of whole runs (host driver included), best of 3",
           "blocks_per_step_max": max(res.blocks_per_step), "block_dim_max": max(res.max_dim_per_step),
           "device_phases_ms_per_run": {k: v[0] / 4 for k, v in phases.items() if v[1]},
           "kernel_launches_per_step": sum(v[1] for v in phases.values()) / 4 / d.nmax,
           "eigenvectors_via_host_bytes": max(spilled),
           "per_block_gpu": {"steps_per_s": d.nmax / t_pb, "ms_per_run": t_pb * 1e3,
                             "impl": "same driver, torch.linalg.eigh (cuSOLVER) one block per launch"}}
    td = np.array(res.td)

    def tddiff(other):
        """Largest relative difference over the values of size 1e-6 or more (values that
        vanish by particle-hole symmetry are round-off noise of order 1e-13 in every run)."""
        o = np.array(other)
        big = np.abs(td) >= 1e-6
        return float(np.max(np.abs(o[big] - td[big]) / np.abs(td[big])))
    out["per_block_gpu"]["td_max_rel_diff"] = tddiff(res_pb.td)

    def specdiff(other):
        """Largest difference of the A_d-A_d spectrum relative to its peak."""
        a, b = res.spectra[C0_SPEC][:, 1], np.asarray(other[C0_SPEC])[:, 1]
        return float(np.max(np.abs(a - b)) / np.max(np.abs(a)))
    out["per_block_gpu"]["spectrum_max_diff_rel_to_peak"] = specdiff(res_pb.spectra)
    out["spectrum_points"] = int(len(res.spectra[C0_SPEC]))
    if not args.no_cpu:
        from oracle import oracle as O
        from oracle import nrg_run_cpu
        O.build()
        threads = os.cpu_count() or 1
        nrg_run_cpu.run(param, data, threads=threads, spectra={})
        spec_cpu = {}
        t0 = time.perf_counter()
        _, td_cpu, _, _ = nrg_run_cpu.run(param, data, threads=threads, spectra=spec_cpu)
        t_cpu = time.perf_counter() - t0
        out["cpu_baseline"] = {"steps_per_s": d.nmax / t_cpu, "ms_per_run": t_cpu * 1e3, "cores": threads,
                               "kind": "port", "sample": "one whole run (thermodynamics and DM-NRG spectrum)",
                               "td_max_rel_diff": tddiff(td_cpu),
                               "spectrum_max_diff_rel_to_peak": specdiff(spec_cpu)}
    return out


def e2e_arm(torch, ctx, hostH, sizes, offs, voffs, args, dist=None, dev=None) -> dict:
    """Same metric through the host-pointer entry point, from pinned host memory (hostH, the
    step's blocks): each step copies the blocks in and the eigenpairs out, streamed through
    the context's bounded device ring (nrg_diag_batch_host returns when they are in host
    memory). Timed with CUDA events around the synchronous calls, after a barrier
    under torchrun; the whole-job value uses the slowest rank's time. Every rank takes the
    same collective steps whether or not its own calls failed."""
    import ctypes as C
    nbk = len(sizes)
    world = dist.get_world_size() if dist else 1
    k = max(1, min(args.steps, 3))
    err, dt = None, math.inf
    try:
        hostV = torch.empty(hostH.numel(), dtype=torch.float64, pin_memory=True)
        hostE = torch.empty(int(voffs[-1]), dtype=torch.float64, pin_memory=True)
        n_c = (C.c_int * nbk)(*[int(x) for x in sizes])
        Hp = (C.c_void_p * nbk)(*[hostH.data_ptr() + 8 * int(offs[b]) for b in range(nbk)])
        Vp = (C.c_void_p * nbk)(*[hostV.data_ptr() + 8 * int(offs[b]) for b in range(nbk)])
        Ep = (C.c_void_p * nbk)(*[hostE.data_ptr() + 8 * int(voffs[b]) for b in range(nbk)])
        info = (C.c_int * nbk)()

        def call():
            rc = ctx.lib.nrg_diag_batch_host(ctx.ptr, nbk, n_c, Hp, Ep, Vp, info, None)
            if rc != 0:
                raise RuntimeError(f"nrg_diag_batch_host returned {rc}")
        call()  # warm-up
    except (RuntimeError, MemoryError) as e:
        err = str(e)[:300]
    if dist:
        dist.barrier()
    if err is None:
        try:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(k):
                call()
            e1.record()
            torch.cuda.synchronize()
            dt = e0.elapsed_time(e1) / 1e3 / k
        except (RuntimeError, MemoryError) as e:
            err = str(e)[:300]
    dt = max_over_ranks(dist, dt, dev)
    out = {"value": world * f_eig(sizes) / dt / 1e9 if math.isfinite(dt) else None, "unit": UNIT,
           "h2d_bytes_per_step": int(8 * offs[-1]) * world,
           "d2h_bytes_per_step": int(8 * (offs[-1] + voffs[-1])) * world, "steps": k,
           "ms_per_step": dt * 1e3 if math.isfinite(dt) else None}
    if err is not None:
        out["error"] = err
    elif not math.isfinite(dt):
        out["error"] = "another rank's host-API calls failed"
    return out


if __name__ == "__main__":
    main()
