"""Sign- and degeneracy-invariant comparison of eigendecompositions (test helper).

Eigenvalues must agree with the oracle's dsyev within 1e-12 * ||H||_2. Eigenvectors are
compared through cluster projectors: eigenvalues closer than 1e-8 * ||H|| form one
cluster, and for every cluster C the projectors V_C^T V_C of both solutions must agree
entrywise within 1e-9. In addition each solution must satisfy the reference's own
is_unitary() tolerances (c++/numerics.hpp:340-367: normalisation 1e-12, orthogonality
1e-10) and have residuals ||H v - lambda v|| <= 1e-12 * ||H|| * sqrt(n).
"""
import numpy as np

VAL_TOL = 1e-12
CLUSTER_REL = 1e-8
PROJ_TOL = 1e-9


def full_from_upper(h: np.ndarray) -> np.ndarray:
    u = np.triu(h)
    return u + np.triu(u, 1).T


def clusters(w: np.ndarray, scale: float):
    out, start = [], 0
    for i in range(1, len(w) + 1):
        if i == len(w) or w[i] - w[i - 1] > CLUSTER_REL * scale:
            out.append((start, i))
            start = i
    return out


def check_eig(h, w, v, w_ref, v_ref, oracle=None):
    H = full_from_upper(np.asarray(h, dtype=np.float64))
    n = H.shape[0]
    nrm = max(np.linalg.norm(H, 2), np.finfo(float).tiny)
    assert w.shape == (n,) and v.shape == (n, n)
    assert np.all(np.diff(w) >= 0), "eigenvalues not ascending"
    dv = np.max(np.abs(w - w_ref))
    assert dv <= VAL_TOL * nrm, f"eigenvalue error {dv:.3e} > {VAL_TOL:.0e}*||H|| ({nrm:.3e})"
    res = np.linalg.norm(v @ H - w[:, None] * v, axis=1).max()
    assert res <= 1e-12 * nrm * max(1.0, np.sqrt(n)), f"residual {res:.3e}"
    if oracle is not None:
        assert oracle.is_unitary(v), "is_unitary() fails"
    else:
        g = v @ v.T
        assert np.abs(np.diag(g) - 1).max() < 1e-12 and np.abs(g - np.diag(np.diag(g))).max() < 1e-10
    worst = 0.0
    for a, b in clusters(w_ref, nrm):
        P = v[a:b].T @ v[a:b]
        Pr = v_ref[a:b].T @ v_ref[a:b]
        worst = max(worst, float(np.abs(P - Pr).max()))
    assert worst <= PROJ_TOL, f"projector difference {worst:.3e} > {PROJ_TOL:.0e}"
    return dv / nrm, worst
