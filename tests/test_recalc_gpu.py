"""Parity of the batched GEMM leaves (C-ABI nrg_gemm3_batch[_host]) with the oracle's
product / transform / rotate (c++/numerics_ublas.hpp:108-140)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-13  # FP64, same association as the reference; only summation order differs


@pytest.fixture(scope="module")
def nb():
    import nrgljubljana_b200 as m
    m.context()
    return m


def close(a, b, rel=REL):
    scale = max(1.0, float(np.abs(b).max()))
    return float(np.abs(a - b).max()) <= rel * scale * max(1, a.size) ** 0.5


def test_all_ones_kats(nb):
    # test/unit/numerics/numerics.cpp:491-520 through the C-ABI
    one = np.ones((2, 2))
    r = np.zeros((2, 2)); nb.product(r, 1.0, one, one); assert (r == 2).all()
    r = np.zeros((2, 2)); nb.transform(r, 1.0, one, one, one); assert (r == 4).all()
    r = np.zeros((2, 2)); nb.rotate(r, 1.0, one, one); assert (r == 4).all()


@pytest.mark.parametrize("dims", [(1, 1, 1, 1), (5, 7, 3, 4), (64, 64, 64, 64), (65, 130, 33, 70), (300, 200, 150, 250)])
def test_transform_strided_views(nb, oracle, dims):
    m, n, ka, kb = dims
    rng = np.random.default_rng(sum(dims))
    # U blocks are column slices of a wider eigenvector matrix (recalc.hpp:18-30)
    U1 = rng.standard_normal((m, ka + 9))[:, 4:4 + ka]
    Up = rng.standard_normal((n, kb + 5))[:, 2:2 + kb]
    O = rng.standard_normal((ka, kb))
    M0 = rng.standard_normal((m, n))
    ref = M0.copy(); oracle.transform(ref, 0.75, np.ascontiguousarray(U1), O, np.ascontiguousarray(Up))
    got = M0.copy(); nb.transform(got, 0.75, U1, O, Up)
    assert close(got, ref)
    ref = M0.copy(); oracle.product(ref, -1.25, np.ascontiguousarray(U1[:, :min(ka, kb)]),
                                    np.ascontiguousarray(Up[:, :min(ka, kb)]))
    got = M0.copy(); nb.product(got, -1.25, U1[:, :min(ka, kb)], Up[:, :min(ka, kb)])
    assert close(got, ref)


@pytest.mark.parametrize("k,d", [(3, 2), (40, 70), (129, 65)])
def test_rotate(nb, oracle, k, d):
    rng = np.random.default_rng(k * 100 + d)
    U = rng.standard_normal((k, d + 3))[:, 1:1 + d]
    R = rng.standard_normal((k, k)); R = R + R.T
    M0 = rng.standard_normal((d, d))
    ref = M0.copy(); oracle.rotate(ref, 0.5, np.ascontiguousarray(U), R)
    got = M0.copy(); nb.rotate(got, 0.5, U, R)
    assert close(got, ref)


def test_batched_terms_accumulate_per_output(nb, oracle):
    """One recalc_general-like call: several table rows add into the same cn (recalc.hpp:97-105)
    and several outputs are computed in the same launch, on device tensors."""
    import torch
    rng = np.random.default_rng(21)
    dims = [37, 80, 12]
    U = [rng.standard_normal((d, 2 * d)) for d in dims]  # eigenvector rows x basis
    terms, refs, outs = [], [], []
    for o in range(4):
        i1, ip = o % 3, (o + 1) % 3
        M = np.zeros((dims[i1], dims[ip]))
        ref = M.copy()
        dev_M = torch.tensor(M, device="cuda")
        for row in range(3):
            c1, cp = row % 2, (row + 1) % 2
            A = U[i1][:, c1 * dims[i1] // 2: c1 * dims[i1] // 2 + 7]
            B = U[ip][:, cp * dims[ip] // 2: cp * dims[ip] // 2 + 5]
            O = rng.standard_normal((7, 5))
            f = float(rng.standard_normal())
            oracle.transform(ref, f, np.ascontiguousarray(A), O, np.ascontiguousarray(B))
            tA, tB, tO = (torch.tensor(np.ascontiguousarray(x), device="cuda") for x in (A, B, O))
            outs.append((tA, tB, tO))
            terms.append(nb.gemm3(dev_M, f, tA, tO, tB))
        refs.append((dev_M, ref))
    nb.gemm3_batch(terms, host=False)
    torch.cuda.synchronize()
    for dev_M, ref in refs:
        assert close(dev_M.cpu().numpy(), ref)


def test_terms_beyond_the_workspace_run_in_passes(nb, oracle):
    """A context whose workspace limit holds the intermediates of a few terms only: the batch
    runs in passes (whole output groups, and the terms of a group too large for one pass), and
    every output gets the same sums; a single term larger than the limit is refused."""
    import torch
    rng = np.random.default_rng(33)
    ctx = nb.Context(workspace_limit=200 * 64 * 8)  # T of three 64 x 64 terms at most
    terms, refs, keep = [], [], []
    for o, nrow in enumerate([1, 2, 7, 3]):  # the 7-term group does not fit in one pass
        M = rng.standard_normal((48, 64))
        ref = M.copy()
        dev_M = torch.tensor(M, device="cuda")
        for row in range(nrow):
            A = rng.standard_normal((64, 48))
            B = rng.standard_normal((64, 64))
            O = rng.standard_normal((64, 64)) if row % 3 else np.diag(rng.standard_normal(64))
            f = float(rng.standard_normal())
            oracle.transform(ref, f, A.T.copy(), O, B)
            tA, tB, tO = (torch.tensor(x, device="cuda") for x in (A, B, O))
            if row % 3 == 0:  # a diagonal O (ldo = 0): the row-scale path
                tO = torch.diagonal(tO).contiguous()
                t = nb.gemm3(dev_M, f, tA, None, tB, transA=True)
                t.O, t.ldo = tO.data_ptr(), 0
            else:
                t = nb.gemm3(dev_M, f, tA, tO, tB, transA=True)
            keep.append((tA, tB, tO))
            terms.append(t)
        refs.append((dev_M, ref))
    nb.gemm3_batch(terms, host=False, ctx=ctx)
    torch.cuda.synchronize()
    for dev_M, ref in refs:
        assert close(dev_M.cpu().numpy(), ref)
    big = torch.zeros((300, 300), dtype=torch.float64, device="cuda")
    with pytest.raises(nb.NRGError):
        nb.gemm3_batch([nb.gemm3(big, 1.0, big, big, big)], host=False, ctx=ctx)


def test_empty_terms_are_skipped(nb):
    M = np.ones((3, 3))
    nb.transform(M, 2.0, np.zeros((3, 0)), np.zeros((0, 0)), np.zeros((3, 0)))
    assert (M == 1).all()


def test_nonfinite_factor_rejected(nb):
    M = np.zeros((2, 2))
    with pytest.raises(nb.NRGError):
        nb.product(M, float("nan"), np.ones((2, 2)), np.ones((2, 2)))
