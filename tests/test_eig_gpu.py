"""Parity of the batched GPU eigensolver (C-ABI nrg_diag_batch[_host]) with the oracle's
LAPACK dsyev (c++/diag.hpp:62-82), through sign/degeneracy-invariant checks."""
import math

import numpy as np
import pytest

from eigcheck import check_eig, full_from_upper

pytestmark = pytest.mark.gpu

SQ2 = 1.0 / math.sqrt(2.0)


@pytest.fixture(scope="module")
def nb():
    import nrgljubljana_b200 as m
    m.context()
    return m


def rand_upper(rng, n, scale=1.0):
    a = rng.standard_normal((n, n)) * scale
    return np.triu(a + a.T)


def graded_block(rng, n):
    """Diagonal 2^{-k/2} plus symmetric N(0, 0.1^2) couplings (the synthetic NRG-like blocks)."""
    h = np.triu(rng.standard_normal((n, n)) * 0.1, 1)
    h[np.diag_indices(n)] = 2.0 ** (-np.arange(n) / 2.0)
    return h


def test_pauli_kats(nb):
    # test/unit/diag_test/diag_test.cpp:83-112 through the C-ABI
    r = nb.diagonalise(np.array([[-1.0, 0.0], [0.0, 1.0]]))
    assert r.val[0] == -1.0 and r.val[1] == 1.0
    assert abs(abs(r.vec[0, 0]) - 1) < 1e-15 and r.vec[0, 1] == 0.0 and r.vec[1, 0] == 0.0
    r = nb.diagonalise(np.array([[0.0, 1.0], [0.0, 0.0]]))
    assert abs(r.val[0] + 1) < 4e-16 and abs(r.val[1] - 1) < 4e-16
    for k in range(2):
        assert abs(abs(r.vec[k, 0]) - SQ2) < 4e-16 and abs(abs(r.vec[k, 1]) - SQ2) < 4e-16
    assert abs(r.vec[0, 0] * r.vec[0, 1] + 0.5) < 4e-16
    assert abs(r.vec[1, 0] * r.vec[1, 1] - 0.5) < 4e-16


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 16, 31, 32, 33, 47, 63, 64])
def test_small_path_random(nb, oracle, n):
    rng = np.random.default_rng(100 + n)
    blocks = [rand_upper(rng, n) for _ in range(3)]
    got = nb.diagonalisations(blocks)
    for h, g in zip(blocks, got):
        w, v = oracle.diagonalise(h)
        check_eig(h, g.val, g.vec, w, v, oracle)


@pytest.mark.parametrize("n", [65, 66, 96, 100, 127, 128, 129, 200, 224, 225, 256, 300, 320, 321, 452, 453,
                               511, 512, 600, 601, 777])
def test_large_path_random(nb, oracle, n):
    rng = np.random.default_rng(200 + n)
    h = rand_upper(rng, n)
    g = nb.diagonalisations([h])[0]
    w, v = oracle.diagonalise(h)
    check_eig(h, g.val, g.vec, w, v, oracle)


@pytest.mark.parametrize("n", [40, 70, 150, 300, 600])
def test_graded_blocks(nb, oracle, n):
    rng = np.random.default_rng(300 + n)
    h = graded_block(rng, n)
    g = nb.diagonalisations([h])[0]
    w, v = oracle.diagonalise(h)
    check_eig(h, g.val, g.vec, w, v, oracle)


@pytest.mark.parametrize("n", [10, 80, 200, 300, 400, 550])
def test_degenerate_spectrum(nb, oracle, n):
    # Exactly repeated eigenvalues (a rotated matrix with a 3-fold and a 5-fold level) and
    # a diagonal matrix: exercises deflation by small z and by close poles.
    rng = np.random.default_rng(400 + n)
    lam = np.sort(rng.standard_normal(n))
    lam[1:4] = lam[1]
    lam[n // 2:n // 2 + 5] = lam[n // 2]
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    H = (q * lam) @ q.T
    h = np.triu(H)
    g = nb.diagonalisations([h])[0]
    w, v = oracle.diagonalise(h)
    check_eig(h, g.val, g.vec, w, v, oracle)
    d = np.triu(np.diag(rng.standard_normal(n)))
    g = nb.diagonalisations([d])[0]
    w, v = oracle.diagonalise(d)
    check_eig(d, g.val, g.vec, w, v, oracle)


@pytest.mark.parametrize("n", [160, 350, 520])
def test_block_diagonal_and_tridiagonal(nb, oracle, n):
    rng = np.random.default_rng(5 + n)
    h = np.zeros((n, n))
    h[:n // 2, :n // 2] = rand_upper(rng, n // 2)
    h[n // 2:, n // 2:] = rand_upper(rng, n - n // 2)  # decoupled halves: beta = 0 at the top split
    h = np.triu(h)
    g = nb.diagonalisations([h])[0]
    w, v = oracle.diagonalise(h)
    check_eig(h, g.val, g.vec, w, v, oracle)
    t = np.diag(rng.standard_normal(n)) + np.diag(rng.standard_normal(n - 1), 1)
    g = nb.diagonalisations([t])[0]
    w, v = oracle.diagonalise(t)
    check_eig(t, g.val, g.vec, w, v, oracle)


def test_mixed_batch(nb, oracle):
    rng = np.random.default_rng(11)
    sizes = [3, 150, 64, 65, 17, 400, 1, 90, 230, 590, 330]
    blocks = [rand_upper(rng, n) if i % 2 else graded_block(rng, n) for i, n in enumerate(sizes)]
    got = nb.diagonalisations(blocks)
    for h, g in zip(blocks, got):
        w, v = oracle.diagonalise(h)
        check_eig(h, g.val, g.vec, w, v, oracle)


def test_device_api_consumes_input(nb, oracle):
    import torch
    rng = np.random.default_rng(12)
    hs = [rand_upper(rng, n) for n in (20, 130)]
    H = [torch.tensor(h, device="cuda") for h in hs]
    E = [torch.empty(h.shape[0], dtype=torch.float64, device="cuda") for h in hs]
    V = [torch.empty_like(x) for x in H]
    info = nb.diag_batch_device(H, E, V)
    torch.cuda.synchronize()
    assert (info == 0).all()
    for h, e, v in zip(hs, E, V):
        w, z = oracle.diagonalise(h)
        check_eig(h, e.cpu().numpy(), v.cpu().numpy(), w, z, oracle)


def test_nonfinite_input_is_reported(nb):
    h = np.eye(5)
    h[0, 3] = np.nan
    with pytest.raises(RuntimeError, match="INFO"):
        nb.diagonalisations([h])
    h = np.triu(np.ones((70, 70)))
    h[10, 20] = np.inf
    with pytest.raises(RuntimeError, match="INFO"):
        nb.diagonalisations([h])


def test_lower_triangle_is_ignored_and_checked(nb):
    rng = np.random.default_rng(13)
    h = rand_upper(rng, 9)
    with pytest.raises(AssertionError):
        nb.diagonalisations([h + np.tril(np.ones((9, 9)), -1)])
    a = nb.diagonalisations([h + np.tril(np.ones((9, 9)), -1)], check_upper=False)[0]
    b = nb.diagonalisations([h])[0]
    assert np.array_equal(a.val, b.val)


def test_dsyevr_ratio(nb, oracle):
    rng = np.random.default_rng(14)
    h = rand_upper(rng, 30)
    r = nb.diagonalise(h, "dsyevr", 0.5)
    w, v = oracle.diagonalise(h, "dsyevr", 0.5)
    assert len(r.val) == len(w) == 15
    assert np.abs(r.val - w).max() < 1e-12 * np.linalg.norm(full_from_upper(h), 2)


@pytest.mark.parametrize("n,kind", [(4097, "random"), (6000, "graded"), (10240, "random")])
def test_large_orders(nb, n, kind):
    """Orders above 4096, where the merge prep of the divide and conquer keeps its arrays in
    global scratch: eigenvalues against host LAPACK (eigvalsh), residuals and orthogonality
    of the vectors computed on the device."""
    import torch
    rng = np.random.default_rng(300 + n)
    h = rand_upper(rng, n) if kind == "random" else graded_block(rng, n)
    g = nb.diagonalisations([h])[0]
    H = full_from_upper(h)
    w_ref = np.linalg.eigvalsh(H)
    nrm = max(abs(w_ref[0]), abs(w_ref[-1]))
    assert np.all(np.diff(g.val) >= 0)
    assert np.max(np.abs(g.val - w_ref)) <= 1e-12 * nrm * max(1.0, math.sqrt(n / 1000.0))
    Hd = torch.tensor(H, device="cuda")
    V = torch.tensor(g.vec, device="cuda")
    w = torch.tensor(g.val, device="cuda")
    res = torch.linalg.norm(V @ Hd - w[:, None] * V, dim=1).max().item()
    assert res <= 1e-12 * nrm * math.sqrt(n)
    G = V @ V.T
    assert (torch.diagonal(G) - 1).abs().max().item() < 1e-12
    assert (G - torch.diag(torch.diagonal(G))).abs().max().item() < 1e-10


@pytest.mark.parametrize("per_sm", [3, 2])
def test_several_reduction_ctas_per_sm(nb, per_sm):
    """1400 blocks of order 601-700: enough streamed blocks for three waves of three (or two)
    CTAs per SM, the launch the benchmark's batch gets (three: two slabs per warp, 168
    registers). Every block's residual and orthogonality are checked on the device."""
    import torch
    ctx = nb.Context()
    ctx.set_tuning(reduction_ctas_per_sm=per_sm)
    g = torch.Generator(device="cuda").manual_seed(93)
    sizes = [601 + (i * 41) % 100 for i in range(1400)]
    H, E, V, H0 = [], [], [], []
    for n in sizes:
        a = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
        h = torch.triu(a + a.T)
        H0.append(h.clone())
        H.append(h)
        E.append(torch.empty(n, dtype=torch.float64, device="cuda"))
        V.append(torch.empty(n, n, dtype=torch.float64, device="cuda"))
    info = nb.diag_batch_device(H, E, V, ctx=ctx)
    torch.cuda.synchronize()
    assert (info == 0).all()
    for h, e, v in zip(H0, E, V):
        n = h.shape[0]
        Hf = h + torch.triu(h, 1).T
        nrm = e.abs().max().item()
        assert torch.linalg.norm(v @ Hf - e[:, None] * v, dim=1).max().item() <= 1e-12 * nrm * math.sqrt(n), n
        assert (v @ v.T - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max().item() < 1e-10, n


def test_few_large_blocks_batch(nb):
    """A batch like a step of the two-channel Kondo runs: a few large blocks, each reduced by
    its own cluster of CTAs at the same time, beside mid-size and small ones."""
    import torch
    rng = np.random.default_rng(77)
    sizes = [3000, 2500, 1800, 1200, 900, 700, 650, 601, 400, 230, 64, 10]
    blocks = [graded_block(rng, n) if i % 2 else rand_upper(rng, n) for i, n in enumerate(sizes)]
    got = nb.diagonalisations(blocks)
    for h, g in zip(blocks, got):
        n = h.shape[0]
        H = full_from_upper(h)
        w_ref = np.linalg.eigvalsh(H)
        nrm = max(abs(w_ref[0]), abs(w_ref[-1]))
        assert np.max(np.abs(g.val - w_ref)) <= 1e-12 * nrm * max(1.0, math.sqrt(n / 1000.0)), n
        Hd = torch.tensor(H, device="cuda")
        V = torch.tensor(g.vec, device="cuda")
        w = torch.tensor(g.val, device="cuda")
        assert torch.linalg.norm(V @ Hd - w[:, None] * V, dim=1).max().item() <= 1e-12 * nrm * math.sqrt(n), n
        G = V @ V.T
        assert (G - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max().item() < 1e-10, n


def test_more_reduction_ctas_than_sms(nb):
    """320 blocks of order 250-900 in one call: with this many the large-block reductions all
    run on the one-CTA bulk-copy kernel, more CTAs than the GPU has SMs (two waves). Every
    block's residual and orthogonality are checked on the device."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(91)
    sizes = [250 + (i * 37) % 651 for i in range(320)]
    H, E, V, H0 = [], [], [], []
    for n in sizes:
        a = torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64)
        h = torch.triu(a + a.T)
        H0.append(h.clone())
        H.append(h)
        E.append(torch.empty(n, dtype=torch.float64, device="cuda"))
        V.append(torch.empty(n, n, dtype=torch.float64, device="cuda"))
    info = nb.diag_batch_device(H, E, V)
    torch.cuda.synchronize()
    assert (info == 0).all()
    for h, e, v in zip(H0, E, V):
        n = h.shape[0]
        Hf = h + torch.triu(h, 1).T
        nrm = e.abs().max().item()
        assert torch.linalg.norm(v @ Hf - e[:, None] * v, dim=1).max().item() <= 1e-12 * nrm * math.sqrt(n), n
        assert (v @ v.T - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max().item() < 1e-10, n
