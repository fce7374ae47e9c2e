"""Parity of the two-stage reduction (dense -> band on the FP64 tensor cores, band ->
tridiagonal by pipelined bulge chasing, both back-transforms) with the oracle's LAPACK dsyev
(c++/diag.hpp:62-82), through the same sign- and degeneracy-invariant checks as the one-stage
path: eigenvalues within 1e-12 ||H||, cluster projectors within 1e-9, residuals and the
reference's is_unitary tolerances."""
import numpy as np
import pytest

from eigcheck import check_eig

pytestmark = pytest.mark.gpu


def two_stage_context(max_blocks=16):
    import nrgljubljana_b200 as nb
    ctx = nb.Context()
    ctx.set_tuning(band_min_n=256, band_max_blocks=max_blocks)
    return ctx


def rand_upper(rng, n):
    a = rng.standard_normal((n, n))
    return np.triu(a + a.T)


def graded_block(rng, n):
    h = np.triu(rng.standard_normal((n, n)) * 0.1, 1)
    h[np.diag_indices(n)] = 2.0 ** (-np.arange(n) / 2.0)
    return h


@pytest.mark.parametrize("n", [256, 257, 290, 300, 513, 640, 1100, 2049])
def test_two_stage_random(oracle, n):
    import nrgljubljana_b200 as nb
    ctx = two_stage_context()
    rng = np.random.default_rng(300 + n)
    h = rand_upper(rng, n)
    g = nb.diagonalisations([h], ctx=ctx)[0]
    w, v = oracle.diagonalise(h)
    check_eig(h, g.val, g.vec, w, v, oracle)


def test_two_stage_structured(oracle):
    """Graded NRG-like blocks, a diagonal matrix (every reflector is the identity), two
    decoupled halves, and an exactly degenerate spectrum."""
    import nrgljubljana_b200 as nb
    ctx = two_stage_context()
    rng = np.random.default_rng(77)
    blocks = [graded_block(rng, 700), np.diag(rng.standard_normal(400))]
    a, b = rand_upper(rng, 200), rand_upper(rng, 230)
    split = np.zeros((430, 430))
    split[:200, :200], split[200:, 200:] = a, b
    blocks.append(split)
    q, _ = np.linalg.qr(rng.standard_normal((360, 360)))
    d = np.repeat([-1.0, 0.5, 2.0], 120)
    blocks.append(np.triu(q @ np.diag(d) @ q.T))
    got = nb.diagonalisations(blocks, ctx=ctx)
    for h, g in zip(blocks, got):
        w, v = oracle.diagonalise(h)
        check_eig(h, g.val, g.vec, w, v, oracle)


def test_two_stage_beside_one_stage(oracle):
    """A batch with three two-stage blocks and one-stage blocks of every other path; the
    result per block is the same as with the two-stage path off, to round-off."""
    import nrgljubljana_b200 as nb
    rng = np.random.default_rng(99)
    sizes = [1200, 900, 700, 600, 450, 300, 200, 120, 64, 20, 5]
    blocks = [rand_upper(rng, n) for n in sizes]
    ctx = two_stage_context(max_blocks=3)
    ctx.set_tuning(band_min_n=700)
    got = nb.diagonalisations(blocks, ctx=ctx)
    off = nb.diagonalisations(blocks, ctx=nb.Context())
    for h, g, o in zip(blocks, got, off):
        w, v = oracle.diagonalise(h)
        check_eig(h, g.val, g.vec, w, v, oracle)
        assert np.abs(g.val - o.val).max() <= 1e-12 * max(1.0, np.abs(o.val).max())


def test_two_stage_off_when_blocks_are_many(oracle):
    """Above band_max_blocks such blocks the batch stays on the one-stage path (the
    throughput regime); the results pass the same bar."""
    import nrgljubljana_b200 as nb
    ctx = two_stage_context(max_blocks=2)
    rng = np.random.default_rng(5)
    blocks = [rand_upper(rng, n) for n in (500, 400, 300)]
    got = nb.diagonalisations(blocks, ctx=ctx)
    for h, g in zip(blocks, got):
        w, v = oracle.diagonalise(h)
        check_eig(h, g.val, g.vec, w, v, oracle)
