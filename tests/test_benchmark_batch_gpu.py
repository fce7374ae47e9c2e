"""The benchmark's whole batched-eigensolve step against the oracle.

All 10,000 blocks of the timed workload (orders log-uniform in [8, 2048], the same seeded
blocks `bench.py` times) are solved in one `nrg_diag_batch` call, so that every block takes the
path and the launch the benchmark measures (three streaming-reduction CTAs per SM, one wave
of the small-block and mid-size paths beside it). A stratified sample of the blocks (every
83rd in size order, 121 blocks of order 8 to 2008) is compared with the oracle's LAPACK
dsyev (c++/diag.hpp:62-82): eigenvalues within 1e-12 ||H||, residuals within
1e-12 ||H|| sqrt(n), orthonormal eigenvectors, and, for the blocks up to order 400, the cluster
projectors within 1e-9 (the sign- and degeneracy-invariant check of the other eigensolver
tests)."""
import math
import os

import numpy as np
import pytest

from eigcheck import VAL_TOL, check_eig

pytestmark = pytest.mark.gpu


def test_benchmark_step_against_oracle(oracle):
    import torch

    import bench
    import nrgljubljana_b200 as nb
    dev = torch.device("cuda", 0)
    sizes = bench.block_sizes(10000, 8, 2048)
    picks = [int(b) for b in np.argsort(sizes, kind="stable")[::83]]
    H = [bench.make_block(torch, b, int(n), dev) for b, n in enumerate(sizes)]
    H0 = {b: H[b].cpu().numpy() for b in picks}
    E = [torch.empty(int(n), dtype=torch.float64, device=dev) for n in sizes]
    V = [torch.empty((int(n), int(n)), dtype=torch.float64, device=dev) for n in sizes]
    info = nb.diag_batch_device(H, E, V)
    torch.cuda.synchronize()
    assert (info == 0).all()
    del H
    w_ref, v_ref = oracle.diag_batch([H0[b] for b in picks], nthreads=os.cpu_count() or 1)
    for k, b in enumerate(picks):
        h, n = H0[b], int(sizes[b])
        w, v = E[b].cpu().numpy(), V[b].cpu().numpy()
        if n <= 400:
            check_eig(h, w, v, w_ref[k], v_ref[k], oracle)
            continue
        Hd = torch.tensor(h, device=dev)
        Hd = Hd + torch.triu(Hd, 1).T
        nrm = float(torch.linalg.matrix_norm(Hd, ord=2))
        assert np.all(np.diff(w) >= 0), n
        assert np.abs(w - w_ref[k]).max() <= VAL_TOL * nrm, n
        vd, wd = V[b], E[b]
        assert torch.linalg.norm(vd @ Hd - wd[:, None] * vd, dim=1).max().item() <= 1e-12 * nrm * math.sqrt(n), n
        assert (vd @ vd.T - torch.eye(n, dtype=torch.float64, device=dev)).abs().max().item() < 1e-10, n
