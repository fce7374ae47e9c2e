"""Serving loop (nrgljubljana_b200.serve): many runs continuously batched into one
eigensolve per tick. Each run's result must be the same alone and in the mix."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
MIX = ["test0_minimal", "legacy_simple", "test13_strategy_all", "test15_safeguard", "test35_betabar",
       "legacy_Himp", "test12_Nmax", "test200_data_has"]


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def test_poisson_arrivals_and_budget_rule():
    from nrgljubljana_b200.nrg_run import RunParams
    from nrgljubljana_b200.serve import poisson_arrivals, run_bytes
    a = poisson_arrivals(200, 4.0, 7)
    assert np.all(np.diff(a) > 0) and np.array_equal(a, poisson_arrivals(200, 4.0, 7))
    assert abs(200 / a[-1] - 4.0) < 1.0
    assert run_bytes(RunParams(keep=2000)) == 4 * run_bytes(RunParams(keep=1000))
    # a run that keeps every step's eigenvectors for its spectra is charged for them
    plain = RunParams(keep=1000)
    spectral = RunParams(keep=1000, dmnrg=True)
    assert run_bytes(spectral, nmax=40) == (3 + 40) * run_bytes(plain, nmax=40) // 3
    assert run_bytes(plain, channels=2) == 16 * run_bytes(plain)


@pytest.fixture(scope="module")
def alone():
    from nrgljubljana_b200.nrg_run import run_files
    return {c: run_files(read(c, "param"), read(c, "data")) for c in MIX}


def same(a, b):
    return (a.td_fields == b.td_fields and a.custom_fields == b.custom_fields
            and np.array_equal(np.array(a.td), np.array(b.td)) and np.array_equal(np.array(a.custom), np.array(b.custom)))


@pytest.mark.gpu
def test_mix_equals_alone(alone):
    from nrgljubljana_b200.serve import Request, Server
    reqs = [Request(i, read(c, "param"), read(c, "data"), 0.0, c) for i, c in enumerate(MIX + MIX[::-1])]
    srv = Server(max_active=16)
    done = srv.serve(reqs, realtime=False)
    assert sorted(d.rid for d in done) == list(range(len(reqs)))
    for d in done:
        assert same(d.result, alone[d.tag]), d.tag
    single = max(max(r.blocks_per_step) for r in alone.values())
    assert max(srv.blocks_per_tick) > single  # the runs shared batched eigensolves


@pytest.mark.gpu
def test_staggered_arrivals_and_tight_budget(alone):
    """Requests arriving while others run join the batch at the next tick; a budget that
    fits one run at a time serialises them; results are unchanged either way."""
    from nrgljubljana_b200.serve import Request, Server
    reqs = [Request(i, read(c, "param"), read(c, "data"), 0.02 * i, c) for i, c in enumerate(MIX)]
    for srv in (Server(max_active=8), Server(hbm_budget=1, max_active=8)):
        done = srv.serve(reqs, realtime=True)
        assert len(done) == len(reqs)
        for d in done:
            assert same(d.result, alone[d.tag]), d.tag
            assert d.done >= d.admitted >= d.arrival - 1e-9


@pytest.mark.gpu
def test_mix_with_large_blocks_within_tolerance():
    """Runs whose blocks reach order ~900: alone, a run's few large blocks are reduced by
    clusters of CTAs, in a tick of twelve runs by the one-CTA kernel. The arithmetic is the
    same with another summation order, so the results agree to round-off (1e-10 relative) as
    long as the truncation keeps the same states. The runs truncate at an energy
    (keepenergy), not at a number of states: a hard cut at `keep` states can fall inside a
    near-degeneracy, where round-off decides which multiplet is kept (as it does between
    LAPACK builds for the reference). Should the kept sets still differ at some step, the
    runs are different calculations from there on and the comparison stops; it must cover
    steps with blocks above order 600."""
    from nrgljubljana_b200.datagen import siam_qs
    from nrgljubljana_b200.nrg_run import run_files
    from nrgljubljana_b200.serve import Request, Server
    reqs = []
    for i in range(12):
        z = 0.1 + 0.075 * i
        param = (f"[param]\nsymtype=QS\nmodel=SIAM\nU=1.0\nGamma=0.05\ndelta=0.05\nband=flat\ndiscretization=Z\n"
                 f"Lambda=2\nz={z!r}\nkeep=10000\nkeepenergy=13\nT=1e-8\nops=n_d\n")
        reqs.append(Request(i, param, siam_qs(1.0, 0.05, 0.05, 2.0, 8, z, "Z", ops=["n_d"]), 0.0, str(i)))
    srv = Server(max_active=16)
    done = srv.serve(reqs, realtime=False)
    assert max(srv.blocks_per_tick) > 100
    for d in done:
        a, m = run_files(reqs[d.rid].param, reqs[d.rid].data), d.result
        # first step whose blocks differ: the kept sets of the step before it differ
        k = next((j for j, (x, y) in enumerate(zip(a.block_dims, m.block_dims)) if x != y), len(a.block_dims))
        assert k >= 4 and max(max(ns) for ns in a.block_dims[:k]) > 600, (d.rid, k)
        # td rows 0..k (calc0 and steps 0..k-1, measured before truncation); custom rows
        # 0..k-1 (measured over the kept states)
        for x, y in ((a.td[:k + 1], m.td[:k + 1]), (a.custom[:k], m.custom[:k])):
            x, y = np.array(x), np.array(y)
            big = np.abs(x) >= 1e-6
            assert np.all(np.abs(x[big] - y[big]) <= 1e-10 * np.abs(x[big])), d.rid
            assert np.all(np.abs(x[~big] - y[~big]) <= 1e-12), d.rid


@pytest.mark.gpu
def test_recalculation_merged_per_tick(alone):
    """Every tick launches the recalculation terms of all active runs in one batched call,
    and the results stay bit for bit those of the runs alone."""
    from nrgljubljana_b200.serve import Request, Server
    reqs = [Request(i, read(c, "param"), read(c, "data"), 0.0, c) for i, c in enumerate(MIX)]
    srv = Server(max_active=8)
    done = srv.serve(reqs, realtime=False)
    # one call per tick that has terms (a tick where every active run ends without operators has none)
    assert srv.ticks - 2 <= srv.recalc_calls <= srv.ticks
    for d in done:
        assert same(d.result, alone[d.tag]), d.tag


@pytest.mark.gpu
def test_spectral_runs_queue_under_a_tight_budget():
    """DM-NRG runs keep every step's eigenvectors for the density matrices; with a budget
    that holds one such run they are served one after another (queued, not out of memory),
    and each result, spectrum included, equals the run alone."""
    from nrgljubljana_b200.inputs import parse_param, read_data
    from nrgljubljana_b200.nrg_run import RunParams, run_files
    from nrgljubljana_b200.serve import Request, Server, run_bytes
    cases = ["test2_algorithms_dmnrg", "test23_DMNRG", "test2_algorithms_dmnrg"]
    charges = [run_bytes(RunParams.from_param(parse_param(read(c, "param"))), read_data(read(c, "data")).nmax)
               for c in cases]
    reqs = [Request(i, read(c, "param"), read(c, "data"), 0.0, c) for i, c in enumerate(cases)]
    srv = Server(hbm_budget=max(charges) + min(charges) - 1, max_active=8)
    done = srv.serve(reqs, realtime=False)
    assert len(done) == len(cases) and srv.max_active_seen == 1
    for d in done:
        a = run_files(read(d.tag, "param"), read(d.tag, "data"))
        assert same(d.result, a), d.tag
        assert sorted(a.spectra) == sorted(d.result.spectra)
        for k in a.spectra:
            # binning sums with FP64 atomics: equal up to the order of the sums (1e-10 of the
            # largest bin, the spectral parity bar)
            x, y = a.spectra[k], d.result.spectra[k]
            assert x.shape == y.shape and np.array_equal(x[:, 0], y[:, 0]), (d.tag, k)
            assert np.abs(x[:, 1] - y[:, 1]).max() <= 1e-10 * np.abs(x[:, 1]).max(), (d.tag, k)
