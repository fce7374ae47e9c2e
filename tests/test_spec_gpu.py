"""Parity of the fused spectral-weight binning (C-ABI nrg_spec_accumulate) with the oracle's
Algo_DMNRG / Algo_FDMgt / Algo_FDMls loops and Bins::add_std (c++/algo_DMNRG.hpp:29-52,
c++/algo_FDM.hpp:30-114, c++/bins.hpp:103-132)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # relative to the largest bin: FP64, atomics change only the summation order


@pytest.fixture(scope="module")
def nb():
    import nrgljubljana_b200 as m
    m.context()
    return m


def rand_energies(rng, n):
    e = 10.0 ** rng.uniform(-11, 0.5, n) * rng.choice([-1.0, 1.0], n)
    e[: max(1, n // 10)] = 0.0 if n > 3 else e[: max(1, n // 10)]
    return np.sort(e)


def sym(rng, k):
    a = rng.standard_normal((k, k)) * 0.1
    return a + a.T


def make_pairs(rng, shapes):
    pairs = []
    for (ni, ki, nj, kj) in shapes:
        pairs.append(dict(Ei=np.abs(rand_energies(rng, ni)), Ej=np.abs(rand_energies(rng, nj)) * 1.3,
                          op1=rng.standard_normal((nj, ni)), op2=rng.standard_normal((nj, ni)),
                          rho_i=sym(rng, ki), rho_j=sym(rng, kj), ki=ki, kj=kj,
                          factor=float(rng.uniform(0.5, 2.0))))
    return pairs


def to_dev(p):
    import torch
    return {k: (torch.tensor(v, device="cuda") if isinstance(v, np.ndarray) else v) for k, v in p.items()}


def compare(cb, pos, neg):
    ref = np.concatenate([cb.pos_re, cb.neg_re])
    got = np.concatenate([pos.cpu().numpy(), neg.cpu().numpy()])
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(cb.pos_im).max() == 0 and np.abs(cb.neg_im).max() == 0
    assert np.abs(got - ref).max() <= TOL * scale, np.abs(got - ref).max() / scale


@pytest.mark.parametrize("bins,lo,hi", [(10, -10.0, 0.0), (1000, -12.0, 2.0)])
def test_dmnrg(nb, oracle, bins, lo, hi):
    import torch
    rng = np.random.default_rng(bins)
    pairs = make_pairs(rng, [(7, 5, 9, 6), (40, 40, 33, 20), (130, 100, 70, 70), (1, 1, 1, 1)])
    grid = nb.BinGrid(lo, hi, bins)
    cb = oracle.ChainBinning(lo, hi, bins)
    Emin, Emax = 1e-9, 5.0
    for p in pairs:
        k = p["ki"]; j = p["kj"]
        cb.dmnrg_pair(p["Ei"][:k], p["Ej"][:j], p["op1"][:j, :k], p["op2"][:j, :k], p["rho_i"], p["rho_j"],
                      p["factor"], -1, Emin, Emax)
    dev = [to_dev(p) for p in pairs]
    descs = [nb.spec_pair(d["Ei"], d["Ej"], d["op1"], d["op2"], d["ki"], d["kj"], d["factor"], d["rho_i"], d["rho_j"])
             for d in dev]
    pos = torch.zeros(grid.nbins, dtype=torch.float64, device="cuda")
    neg = torch.zeros_like(pos)
    nb.spec_accumulate(0, descs, grid, pos, neg, sign=-1, Emin=Emin, Emax=Emax)
    torch.cuda.synchronize()
    compare(cb, pos, neg)


@pytest.mark.parametrize("which", ["gt", "ls"])
def test_fdm(nb, oracle, which):
    import torch
    rng = np.random.default_rng(5 if which == "gt" else 6)
    pairs = make_pairs(rng, [(9, 4, 12, 5), (80, 30, 60, 25), (200, 90, 150, 60)])
    grid = nb.BinGrid(-14.0, 2.0, 100)
    cb = oracle.ChainBinning(-14.0, 2.0, 100)
    T, wnf, sign = 1e-3, 0.37, -1
    for p in pairs:
        rho = p["rho_i"] if which == "gt" else p["rho_j"]
        cb.fdm_pair(which, p["Ei"], p["ki"], p["Ej"], p["kj"], p["op1"], p["op2"], rho, p["factor"], sign, T, wnf)
    dev = [to_dev(p) for p in pairs]
    descs = [nb.spec_pair(d["Ei"], d["Ej"], d["op1"], d["op2"], d["ki"], d["kj"], d["factor"],
                          d["rho_i"] if which == "gt" else None, d["rho_j"] if which == "ls" else None) for d in dev]
    pos = torch.zeros(grid.nbins, dtype=torch.float64, device="cuda")
    neg = torch.zeros_like(pos)
    nb.spec_accumulate(1 if which == "gt" else 2, descs, grid, pos, neg, sign=sign, T=T, wnf=wnf)
    torch.cuda.synchronize()
    compare(cb, pos, neg)


def test_large_grid_uses_global_atomics(nb, oracle):
    # 20 decades at 1000 bins per decade do not fit a private shared-memory histogram
    import torch
    rng = np.random.default_rng(9)
    pairs = make_pairs(rng, [(64, 64, 64, 64)])
    grid = nb.BinGrid(-18.0, 2.0, 1000)
    cb = oracle.ChainBinning(-18.0, 2.0, 1000)
    p = pairs[0]
    cb.dmnrg_pair(p["Ei"], p["Ej"], p["op1"], p["op2"], p["rho_i"], p["rho_j"], p["factor"], 1, 0.0, 1e3)
    d = to_dev(p)
    pos = torch.zeros(grid.nbins, dtype=torch.float64, device="cuda")
    neg = torch.zeros_like(pos)
    nb.spec_accumulate(0, [nb.spec_pair(d["Ei"], d["Ej"], d["op1"], d["op2"], 64, 64, p["factor"], d["rho_i"],
                                        d["rho_j"])], grid, pos, neg, sign=1, Emin=0.0, Emax=1e3)
    torch.cuda.synchronize()
    compare(cb, pos, neg)
