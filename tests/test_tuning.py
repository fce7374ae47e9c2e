"""Launch parameters of the batched eigensolver (nrg_tuning) and the autotuner's table.

Every choice of crossover orders sends blocks down another path (one-CTA solver, one-CTA
or cluster shared-memory reduction, streaming reduction); whatever the choice, the
eigenpairs must pass the same parity bar against the oracle's dsyev."""
import json

import numpy as np
import pytest

from eigcheck import check_eig


def test_table_lookup_by_device_name(tmp_path, monkeypatch):
    from nrgljubljana_b200 import autotune
    tab = {"NVIDIA B200": {"tuning": {"small_max_n": 48, "mid_max_n": 192, "cluster_max_n": 560,
                                      "reduction_ctas_per_sm": 1, "band_min_n": 2048, "band_max_blocks": 8},
                           "objective": 0.9}}
    p = tmp_path / "tuning.json"
    p.write_text(json.dumps(tab))
    monkeypatch.setattr(autotune, "TABLE", str(p))
    monkeypatch.setattr(autotune, "device_name", lambda device=0: "NVIDIA B200")
    assert autotune.load_table(0) == tab["NVIDIA B200"]["tuning"]
    monkeypatch.setattr(autotune, "device_name", lambda device=0: "another device")
    assert autotune.load_table(0) is None


def test_workloads_are_seeded():
    from nrgljubljana_b200 import autotune
    a, b = autotune.workloads(), autotune.workloads()
    assert len(a) == 14 and all(np.array_equal(x, y) for x, y in zip(a, b))
    assert 200 <= a[12].min() and a[12].max() <= 7049
    assert max(int(x.max()) for x in a[:8]) <= 480 and max(int(x.max()) for x in a[8:10]) <= 1024
    assert 800 <= a[10].min() and a[10].max() <= 2000 and 1500 <= a[11].min() and a[11].max() <= 4096
    assert len(a[13]) == 1500 and 8 <= a[13].min() and a[13].max() <= 2048


@pytest.mark.gpu
def test_set_tuning_checks_ranges():
    import nrgljubljana_b200 as nb
    ctx = nb.Context()
    t0 = ctx.tuning
    for bad in ({"small_max_n": 31}, {"small_max_n": 97}, {"mid_max_n": 237}, {"cluster_max_n": 641},
                {"small_max_n": 96, "mid_max_n": 90}, {"reduction_ctas_per_sm": 4}, {"reduction_ctas_per_sm": 0}):
        with pytest.raises(nb.NRGError):
            ctx.set_tuning(**bad)
        assert ctx.tuning == t0
    ctx.set_tuning(small_max_n=96, mid_max_n=236, cluster_max_n=640)
    assert ctx.tuning["small_max_n"] == 96 and ctx.tuning["cluster_max_n"] == 640


@pytest.mark.gpu
@pytest.mark.parametrize("tuning", [dict(small_max_n=32, mid_max_n=128, cluster_max_n=400),
                                    dict(small_max_n=96, mid_max_n=236, cluster_max_n=640),
                                    dict(small_max_n=48, mid_max_n=160, cluster_max_n=480)])
def test_every_path_choice_is_correct(oracle, tuning):
    import nrgljubljana_b200 as nb
    ctx = nb.Context()
    ctx.set_tuning(**tuning)
    rng = np.random.default_rng(4242)
    sizes = [8, 31, 33, 47, 64, 80, 96, 97, 127, 130, 160, 190, 230, 236, 237, 300, 410, 470, 520, 600, 639, 660]
    blocks = []
    for n in sizes:
        a = rng.standard_normal((n, n))
        blocks.append(np.triu(a + a.T))
    got = nb.diagonalisations(blocks, ctx=ctx)
    for h, g in zip(blocks, got):
        w, v = oracle.diagonalise(h)
        check_eig(h, g.val, g.vec, w, v, oracle)
