"""The replica path of bench.py under torchrun, on CPU with gloo (world size 2): every rank
gets the slowest rank's time, also when one rank failed and passed inf, and the reference
arm runs on rank 0 only, the other ranks exiting 0 without output. The end-to-end arm's
control flow (warm-up, timed host-API calls, whole-job value, failure without a number) is
checked with host-only stand-ins for the torch calls and the library."""
import datetime
import math
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VALUES = [[1.5, 2.5], [3.0, math.inf], [0.25, 0.125]]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    got = [bench.max_over_ranks(dist, v[rank], "cpu") for v in VALUES]
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, got))


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [max(v) for v in VALUES]
    assert res[0] == want and res[1] == want


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 2.5, "cpu") == 2.5


def test_reference_arm_only_on_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


class _FakeBuf:
    def __init__(self, n):
        import numpy as np
        self.a = np.zeros(n)

    def numel(self):
        return self.a.size

    def copy_(self, other):
        return self

    def data_ptr(self):
        return self.a.ctypes.data


class _FakeTorch:
    """The few torch calls of bench.e2e_arm, host-only: events report 250 ms between them."""
    float64 = "float64"

    class cuda:
        class Event:
            def __init__(self, enable_timing=True):
                pass

            def record(self):
                pass

            def elapsed_time(self, other):
                return 250.0

        @staticmethod
        def synchronize():
            pass

    @staticmethod
    def empty(n, dtype=None, pin_memory=False):
        return _FakeBuf(n)


class _FakeLib:
    def __init__(self, rc):
        self.rc, self.calls = rc, 0

    def nrg_diag_batch_host(self, *args):
        self.calls += 1
        return self.rc


def _e2e(rc):
    import types

    import numpy as np
    sys.path.insert(0, ROOT)
    import bench
    sizes = np.array([10, 20, 30])
    offs = np.concatenate([[0], np.cumsum(sizes ** 2)])
    voffs = np.concatenate([[0], np.cumsum(sizes)])
    ctx = types.SimpleNamespace(lib=_FakeLib(rc), ptr=None)
    args = types.SimpleNamespace(steps=5)
    out = bench.e2e_arm(_FakeTorch, ctx, _FakeBuf(int(offs[-1])), sizes, offs, voffs, args)
    return bench, sizes, offs, voffs, ctx, out


def test_e2e_arm_reports_host_api_throughput():
    bench, sizes, offs, voffs, ctx, out = _e2e(0)
    assert ctx.lib.calls == 1 + 3  # warm-up, then min(steps, 3) timed calls
    assert out["steps"] == 3 and math.isclose(out["ms_per_step"], 250.0 / 3)
    assert math.isclose(out["value"], bench.f_eig(sizes) / (0.25 / 3) / 1e9)
    assert out["h2d_bytes_per_step"] == 8 * int(offs[-1])
    assert out["d2h_bytes_per_step"] == 8 * int(offs[-1] + voffs[-1])
    assert "error" not in out


def test_e2e_arm_failure_gives_no_number():
    _, _, _, _, ctx, out = _e2e(-7)
    assert ctx.lib.calls == 1 and out["value"] is None and "returned -7" in out["error"]
