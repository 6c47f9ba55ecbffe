"""TEST INFRASTRUCTURE — dense CPU restatement of the reference's CRV3 variance for OLS (numpy),
the checker of the device CRV3 path.

Only tests/ use this module; the product (fereg_b200) never imports it.

CRV3 is the leave-one-cluster-out jackknife (crv3.rs:1-30, pyfixest `_vcov_crv3_slow`): for every
cluster g the model is refitted without g's rows, the fixed effects re-estimated, here as the
weighted least squares on [X, the FE dummies of the remaining rows] (exact, any nesting). With
absorbed terms the constant of a refit is the regression-through-the-means constant of its sample
(ols/stata_vce.rs:572-600 add_constant). The meat is the inclusion-exclusion sum over the non-empty
subsets S of the cluster dimensions of (-1)^(|S|+1) sum_g (theta_(-g) - theta)(theta_(-g) - theta)'
(ols/stata_vce.rs:516-545), theta the full-sample [b, _cons]; V = q meat with reghdfe's cluster
factor q = (N - 1) / (N - nested - df_m - df_a) G_min / (G_min - 1) (ols.rs:417-419, 519); with
several dimensions the eigenvalue clip of vcov.rs:689-710.
"""

import itertools

import numpy as np


def _dense_fit(codes, g, y, X, w):
    """b of y on X with the FE dummies (levels present in the rows) absorbed; weighted."""
    D = np.concatenate([np.eye(gq)[c][:, np.unique(c)] for c, gq in zip(codes, g)], axis=1)
    Z = np.column_stack([X, D])
    sw = np.sqrt(w)
    beta, *_ = np.linalg.lstsq(Z * sw[:, None], y * sw, rcond=None)
    return beta[: X.shape[1]]


def _clip(v):
    lam, u = np.linalg.eigh(v)
    if not (lam < 0).any():
        return None
    lam = np.where(lam > 0, lam, 0.0)
    out = (u * lam) @ u.T
    return (out + out.T) / 2


def fix_psd(v, constant):
    """vcov.rs:689-710: symmetrize, clip the whole; with a constant, the slopes' block clipped on
    its own and written back."""
    v = (v + v.T) / 2
    k = v.shape[0]
    kb = k - 1 if constant else k
    backup = v[:kb, :kb].copy()
    c = _clip(v)
    if c is None:
        return v
    if constant:
        sub = _clip(backup)
        c[:kb, :kb] = backup if sub is None else sub
    return c


def crv3_ols(codes, g, y, X, clusters, df_a, nested, w=None):
    """V of [b (X's columns), _cons] (absorbed terms: the constant reported) and the full-sample
    theta. clusters: list of (codes, G); df_a and nested (df_a_nested > 0) from the dof."""
    y = np.asarray(y, dtype=float)
    X = np.asarray(X, dtype=float)
    n, k = X.shape
    w = np.ones(n) if w is None else np.asarray(w, dtype=float)

    def theta(rows):
        b = _dense_fit([c[rows] for c in codes], g, y[rows], X[rows], w[rows])
        ww = w[rows]
        b0 = (ww @ y[rows] - b @ (ww @ X[rows])) / ww.sum()
        return np.append(b, b0)

    full = theta(np.arange(n))
    meat = np.zeros((k + 1, k + 1))
    for size in range(1, len(clusters) + 1):
        for sub in itertools.combinations(range(len(clusters)), size):
            key = np.zeros(n, dtype=np.int64)
            for d in sub:
                key = key * (clusters[d][1] + 1) + clusters[d][0]
            _, cc = np.unique(key, return_inverse=True)
            sign = 1.0 if size % 2 == 1 else -1.0
            for gg in range(cc.max() + 1):
                d = theta(np.flatnonzero(cc != gg)) - full
                meat += sign * np.outer(d, d)
    gmin = min(G for _, G in clusters)  # N = n: unweighted or aweights
    q = (n - 1) / (n - (1 if nested else 0) - k - df_a) * gmin / (gmin - 1)
    V = q * meat
    if len(clusters) > 1:
        V = fix_psd(V, True)
    return full, V
