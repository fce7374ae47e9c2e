"""The allocation-free transform entry point (nrg_transform_noalloc), called through the
C-ABI and checked against the batched entry point nrg_gemm3_batch on the same inputs.

This file is collected last, so that a run stopping at the first failure has run every
other test before it. It must pass alone in a fresh process as well."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-13  # the tolerance of the GEMM-leaf parity tests


def _view(torch, rng, rows, cols, pad):
    """A strided view (leading dimension cols + 2 * pad) such as a U(i) block of recalc.hpp."""
    wide = torch.tensor(rng.standard_normal((rows, cols + 2 * pad)), device="cuda")
    return wide[:, pad:pad + cols]


def test_noalloc_matches_batched_entry_point_twice():
    import torch

    import nrgljubljana_b200 as nb
    lib = nb.load_library()
    nb.context()
    rng = np.random.default_rng(2027)
    # two calls in a row with different shapes: the shared scratch keeps the first call's
    # contents, which the second call must not depend on
    for rows, cols, ka, kb, f in ((70, 90, 40, 33, 0.75), (33, 129, 64, 17, -1.5)):
        A = _view(torch, rng, rows, ka, 3)
        B = _view(torch, rng, cols, kb, 2)
        O = torch.tensor(rng.standard_normal((ka, kb)), device="cuda")
        M0 = torch.tensor(rng.standard_normal((rows, cols)), device="cuda")
        ref = M0.clone()
        nb.gemm3_batch([nb.gemm3(ref, f, A, O, B)], host=False)
        got = M0.clone()
        rc = lib.nrg_transform_noalloc(got.data_ptr(), got.stride(0), A.data_ptr(), A.stride(0), O.data_ptr(),
                                       O.stride(0), B.data_ptr(), B.stride(0), rows, cols, ka, kb, f, None)
        assert rc == 0, nb._lib.last_error()
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.abs(g - r).max() <= REL * max(1.0, np.abs(r).max()) * g.size ** 0.5
    # identity O (product): no scratch involved
    A = _view(torch, rng, 20, 16, 1)
    B = _view(torch, rng, 24, 16, 1)
    ref = torch.zeros((20, 24), dtype=torch.float64, device="cuda")
    nb.gemm3_batch([nb.gemm3(ref, 2.0, A, None, B)], host=False)
    got = torch.zeros_like(ref)
    assert lib.nrg_transform_noalloc(got.data_ptr(), 24, A.data_ptr(), A.stride(0), None, 0, B.data_ptr(),
                                     B.stride(0), 20, 24, 16, 16, 2.0, None) == 0
    torch.cuda.synchronize()
    assert torch.allclose(got, ref, rtol=REL, atol=REL)


def test_noalloc_at_the_scratch_limit_matches_batched_and_oracle():
    """ka * cols exactly equal to the scratch size is accepted, and every element of the
    intermediate is used: the result equals the batched entry point's and the oracle's
    transform() (c++/numerics_ublas.hpp:119-128)."""
    import torch

    import nrgljubljana_b200 as nb
    from oracle import oracle
    lib = nb.load_library()
    limit = nb._lib.NRG_NOALLOC_SCRATCH_DOUBLES
    ka, cols = 1024, limit // 1024
    assert ka * cols == limit
    rows, kb, f = 24, 12, 0.375
    rng = np.random.default_rng(2028)
    A = torch.tensor(rng.standard_normal((rows, ka)), device="cuda")
    O = torch.tensor(rng.standard_normal((ka, kb)), device="cuda")
    B = torch.tensor(rng.standard_normal((cols, kb)), device="cuda")
    M0 = rng.standard_normal((rows, cols))
    ref = torch.tensor(M0, device="cuda")
    nb.gemm3_batch([nb.gemm3(ref, f, A, O, B)], host=False)
    for _ in range(2):  # two calls in a row on the shared scratch
        got = torch.tensor(M0, device="cuda")
        rc = lib.nrg_transform_noalloc(got.data_ptr(), cols, A.data_ptr(), ka, O.data_ptr(), kb, B.data_ptr(), kb,
                                       rows, cols, ka, kb, f, None)
        assert rc == 0, nb._lib.last_error()
        torch.cuda.synchronize()
        g, r = got.cpu().numpy(), ref.cpu().numpy()
        scale = max(1.0, np.abs(r).max())
        assert np.abs(g - r).max() <= REL * scale * ka ** 0.5
    host = M0.copy()
    oracle.transform(host, f, A.cpu().numpy(), O.cpu().numpy(), B.cpu().numpy())
    assert np.abs(g - host).max() <= REL * max(1.0, np.abs(host).max()) * ka ** 0.5


def test_noalloc_rejects_bad_leading_dimensions():
    """ldo = 0 (the batched API's diagonal O) and leading dimensions shorter than a row are
    rejected, so that no call reads a dense operand with a wrong stride."""
    import torch

    import nrgljubljana_b200 as nb
    lib = nb.load_library()
    rows, cols, ka, kb = 8, 9, 6, 5
    M = torch.zeros((rows, cols), dtype=torch.float64, device="cuda")
    A = torch.zeros((rows, ka), dtype=torch.float64, device="cuda")
    O = torch.zeros((ka, kb), dtype=torch.float64, device="cuda")
    B = torch.zeros((cols, kb), dtype=torch.float64, device="cuda")
    good = dict(ldm=cols, lda=ka, ldo=kb, ldb=kb)
    for key, bad in (("ldo", 0), ("ldo", kb - 1), ("lda", ka - 1), ("ldb", kb - 1), ("ldm", cols - 1)):
        ld = dict(good, **{key: bad})
        rc = lib.nrg_transform_noalloc(M.data_ptr(), ld["ldm"], A.data_ptr(), ld["lda"], O.data_ptr(), ld["ldo"],
                                       B.data_ptr(), ld["ldb"], rows, cols, ka, kb, 1.0, None)
        assert rc == nb._lib.NRG_ERR_ARG, (key, bad)
        assert key in nb._lib.last_error()
    assert lib.nrg_transform_noalloc(M.data_ptr(), cols, A.data_ptr(), ka, O.data_ptr(), kb, B.data_ptr(), kb, rows,
                                     cols, ka, kb, 1.0, None) == 0


def test_noalloc_rejects_sizes_beyond_the_scratch():
    import torch

    import nrgljubljana_b200 as nb
    lib = nb.load_library()
    limit = nb._lib.NRG_NOALLOC_SCRATCH_DOUBLES
    ka, cols = 1024, limit // 1024 + 1
    M = torch.zeros((1, cols), dtype=torch.float64, device="cuda")
    A = torch.zeros((1, ka), dtype=torch.float64, device="cuda")
    O = torch.zeros((ka, 1), dtype=torch.float64, device="cuda")
    B = torch.zeros((cols, 1), dtype=torch.float64, device="cuda")
    rc = lib.nrg_transform_noalloc(M.data_ptr(), cols, A.data_ptr(), ka, O.data_ptr(), 1, B.data_ptr(), 1, 1, cols, ka,
                                   1, 1.0, None)
    assert rc == nb._lib.NRG_ERR_ARG
    assert "static scratch" in nb._lib.last_error()
