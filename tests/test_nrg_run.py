"""Whole NRG runs (symtype QS, one channel) against the reference's regression outputs.

Each case under tests/golden/nrg/ is one of the reference's regression tests
(test/c++/<case>: param, data, ref/td, ref/custom; copied by make_nrg_fixtures.py). The
CPU restatement in oracle/nrg_run_cpu.py is pinned against the printed refs on the CPU;
the device run (nrgljubljana_b200.nrg_run, Hamiltonian assembly + batched eigensolver +
batched recalculation on the GPU) is checked against the refs and against the oracle.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "nrg")
CASES = sorted(os.listdir(GOLD))

# The refs are printed with 10 significant digits (c++/params.hpp:394-396); quantities that
# vanish by symmetry (<Q> at particle-hole symmetry) are round-off noise of order 1e-13.
REF_RTOL, REF_ATOL = 2e-9, 1e-11
# GPU run against the oracle at full precision: different eigensolvers, same physics.
ORA_RTOL, ORA_ATOL = 1e-10, 1e-11


def read(case, name):
    with open(os.path.join(GOLD, case, name)) as f:
        return f.read()


def ref_rows(case, name):
    path = os.path.join(GOLD, case, name)
    if not os.path.exists(path):
        return None, None
    header, rows = None, []
    for line in open(path):
        if line.startswith("#"):
            header = line[1:].split()
        elif line.strip():
            rows.append([float(x) for x in line.split()])
    return header, np.array(rows)


def assert_close(got, want, rtol, atol, what):
    got, want = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    err = np.abs(got - want) - (rtol * np.abs(want) + atol)
    if np.any(err > 0):
        r, c = np.unravel_index(int(np.argmax(err)), err.shape)
        raise AssertionError(f"{what}: row {r} col {c}: {got[r, c]!r} vs {want[r, c]!r}")


@pytest.fixture(scope="module")
def oracle_runs(oracle):
    from oracle import nrg_run_cpu
    cache = {}

    def get(case):
        if case not in cache:
            cache[case] = nrg_run_cpu.run(read(case, "param"), read(case, "data"), threads=os.cpu_count() or 1)
        return cache[case]
    return get


# ------------------------------------------------------------------ CPU: readers and oracle
def test_data_reader_minimal():
    from nrgljubljana_b200.inputs import read_data
    d = read_data(read("test0_minimal", "data"))
    assert (d.symtype, d.channels, d.nmax) == ("QS", 1, 4)
    assert [I for I, _ in d.subspaces] == [(-2, 1), (-1, 2), (0, 1), (0, 3), (1, 2), (2, 1)]
    assert [len(e) for _, e in d.subspaces] == [1, 2, 3, 1, 2, 1]
    assert len(d.opch[0][0]) == 6 and d.opch[0][0][((0, 1), (-1, 2))].shape == (3, 2)
    assert abs(d.gs_energy - (-0.21659058369307171)) < 1e-17
    assert list(d.ops) == ["n_d"] and d.ops["n_d"][0] == "s"
    assert len(d.xi[0]) == 5 and len(d.zeta[0]) == 5
    assert d.xi[0][0] == 0.54528747084262258072 and d.zeta[0][4] == 0.0


def test_param_reader_rejects_unsupported():
    from nrgljubljana_b200.inputs import parse_param
    from nrgljubljana_b200.nrg_run import RunParams
    p = RunParams.from_param(parse_param(read("test15_safeguard", "param")))
    assert (p.keep, p.safeguard, p.Lambda) == (100, 0.1, 2.0)
    for bad in ("Ninit=1", "diagratio=0.1", "substeps=true", "absolute=true", "strategy=some", "specgt=A_d-A_d"):
        with pytest.raises(ValueError):
            RunParams.from_param(parse_param("[param]\n" + bad + "\n"))


def test_param_reader_accepts_every_fixture():
    """Every regression input the GPU tests run is accepted by the driver's parameter reader."""
    from nrgljubljana_b200.inputs import parse_param
    from nrgljubljana_b200.nrg_run import RunParams
    for case in CASES:
        RunParams.from_param(parse_param(read(case, "param")))


def test_cluster_mapping_quirks():
    # c++/splitting.hpp:48-72: split clusters map to their lowest member; the last cluster
    # is never closed, so its members stay as they are.
    from nrgljubljana_b200.nrg_run import cluster_mapping
    e = np.array([0.0, 1.0, 1.0 + 2e-16, 1.0 + 4e-16, 2.0, 3.0, 3.0 + 4e-16])
    m = cluster_mapping(e, 1e-15)
    assert m == {float(e[2]): 1.0, float(e[3]): 1.0}
    assert cluster_mapping(np.array([0.0, 0.0, 1.0]), 1e-15) == {}


def test_highest_retained_energy():
    from nrgljubljana_b200.nrg_run import RunParams, highest_retained_energy
    e = np.array([0.0, 0.1, 0.2, 0.2 + 1e-7, 0.5, 0.9])
    assert highest_retained_energy(e, RunParams(keep=3)) == 0.2 + 1e-7  # safeguard keeps the pair
    assert highest_retained_energy(e, RunParams(keep=3, safeguard=0.0)) == 0.2
    assert highest_retained_energy(e, RunParams(keep=100, keepenergy=0.3, keepmin=0)) == 0.5
    assert highest_retained_energy(e, RunParams(keep=100)) == 0.9


@pytest.mark.parametrize("case", CASES)
def test_oracle_run_matches_reference(oracle_runs, case):
    tdf, td, cf, cu = oracle_runs(case)
    hdr, ref = ref_rows(case, "td")
    assert hdr == tdf
    assert_close(td, ref, REF_RTOL, REF_ATOL, f"{case} td")
    hdr, ref = ref_rows(case, "custom")
    if ref is not None:
        assert hdr == cf
        assert_close(cu, ref, REF_RTOL, REF_ATOL, f"{case} custom")


# ------------------------------------------------------------------ GPU: the device run
@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_run_matches_reference_and_oracle(oracle_runs, case):
    from nrgljubljana_b200.nrg_run import run_files
    res = run_files(read(case, "param"), read(case, "data"))
    hdr, ref = ref_rows(case, "td")
    assert hdr == res.td_fields
    assert_close(res.td, ref, REF_RTOL, REF_ATOL, f"{case} td vs reference")
    tdf, td, cf, cu = oracle_runs(case)
    assert_close(res.td, td, ORA_RTOL, ORA_ATOL, f"{case} td vs oracle")
    hdr, ref = ref_rows(case, "custom")
    if ref is not None:
        assert hdr == res.custom_fields
        assert_close(res.custom, ref, REF_RTOL, REF_ATOL, f"{case} custom vs reference")
    assert_close(res.custom, cu, ORA_RTOL, ORA_ATOL, f"{case} custom vs oracle")


@pytest.mark.gpu
def test_hamiltonian_batch_bitexact():
    """nrg_hamiltonian_batch against the same additions done in numpy, bit for bit: the
    sqrt(Lambda)-scaled ancestor energies, zeta shifts and xi-scaled <||f||> blocks, in
    their order, plus a transposed block and blocks spread over many tiles."""
    import ctypes as C
    import torch
    import nrgljubljana_b200 as m
    from nrgljubljana_b200._lib import HPiece, NRG_HP_BLOCK, NRG_HP_DIAG
    from nrgljubljana_b200.api import _stream_ptr
    ctx = m.context()
    rng = np.random.default_rng(7)
    dev = torch.device("cuda", 0)
    ns = [1, 5, 37, 130, 300]
    Hs = [torch.full((n, n), np.nan, dtype=torch.float64, device=dev) for n in ns]
    want = [np.zeros((n, n)) for n in ns]
    keep = []
    pieces = []
    for b, n in enumerate(ns):
        cut = sorted(rng.choice(np.arange(1, n), size=min(3, n - 1), replace=False)) if n > 1 else []
        offs = [0] + list(cut) + [n]
        dims = [offs[i + 1] - offs[i] for i in range(len(offs) - 1)]
        for i, dd in enumerate(dims):
            v = rng.standard_normal(dd)
            t = torch.from_numpy(v).to(dev)
            keep.append(t)
            f = float(np.sqrt(2.0))
            pieces.append(HPiece(b, NRG_HP_DIAG, offs[i], offs[i], dd, dd, 0, 0, 0, t.data_ptr(), f, 0.0))
            idx = np.arange(offs[i], offs[i] + dd)
            want[b][idx, idx] = f * v
        for i in range(len(dims)):
            for j in range(i + 1, len(dims)):
                trans = (i + j) % 2
                mat = rng.standard_normal((dims[j], dims[i]) if trans else (dims[i], dims[j]))
                wide = rng.standard_normal((mat.shape[0], mat.shape[1] + 3))
                wide[:, :mat.shape[1]] = mat
                t = torch.from_numpy(wide).to(dev)
                keep.append(t)
                fs = float(rng.standard_normal()) / 0.7
                pieces.append(HPiece(b, NRG_HP_BLOCK, offs[i], offs[j], dims[i], dims[j], trans, 0, wide.shape[1],
                                     t.data_ptr(), fs, 0.0))
                want[b][offs[i]:offs[i + 1], offs[j]:offs[j + 1]] += fs * (mat.T if trans else mat)
        for i, dd in enumerate(dims):
            shift = float(rng.standard_normal()) * (2.0 - 1.0) / 0.3
            pieces.append(HPiece(b, NRG_HP_DIAG, offs[i], offs[i], dd, dd, 0, 0, 0, None, 0.0, shift))
            idx = np.arange(offs[i], offs[i] + dd)
            want[b][idx, idx] += shift
    # blocks interleaved round-robin in the array; the order inside each block is kept
    per_block = [[q for q in pieces if q.blk == b] for b in range(len(ns))]
    seq = []
    while any(per_block):
        for lst in per_block:
            if lst:
                seq.append(lst.pop(0))
    arr = (HPiece * len(seq))(*seq)
    n_arr = (C.c_int * len(ns))(*ns)
    Hp = (C.c_void_p * len(ns))(*[h.data_ptr() for h in Hs])
    rc = ctx.lib.nrg_hamiltonian_batch(ctx.ptr, len(ns), n_arr, Hp, len(pieces), arr,
                                       _stream_ptr(torch.cuda.current_stream()))
    assert rc == 0
    torch.cuda.synchronize()
    for b in range(len(ns)):
        got = Hs[b].cpu().numpy()
        assert np.array_equal(got, want[b]), f"block {b}: max diff {np.nanmax(np.abs(got - want[b]))}"
