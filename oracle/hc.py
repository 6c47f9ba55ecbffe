"""TEST INFRASTRUCTURE — dense CPU restatement of the reference's HC2 / HC3 variance for OLS
(numpy), the checker of the device path.

Only tests/ use this module; the product (fereg_b200) never imports it.

Stata `regress ..., vce(hc2|hc3)` with explicit FE dummies (the reference's ols.rs:450-474 with
leverage.rs:128 fe_hat and ols/stata_vce.rs:156-167 hc_mult): b from the weighted least squares
on [X, D] (D: the FE dummies, or the constant without absorbed terms), h_i = w_i z_i'(Z'WZ)^+ z_i
the leverage of the full weighted design, robust scores s_i = e_i w_i, tau_i = w_i with fweights
else 1, HC2 meat sum s^2 / (tau - h) z z', HC3 sum tau s^2 / (tau - h)^2 z z' (rows with
tau - h <= sqrt(eps) tau left out), V = (Z'WZ)^+ meat (Z'WZ)^+ without a small-sample factor.
Weights: aweights and pweights normalized to sum N, fweights as given (ols.rs:77-108).
"""

import numpy as np


def hc_ols(codes, g, y, X, hc3, w=None, weight_kind=None):
    """b and V of [X..., _cons] for absorbed terms (codes non-empty: the constant reported as the
    regression-through-the-means one, V's constant row from the dummies' design) or of
    [X..., _cons] on the plain design when codes is empty."""
    y = np.asarray(y, dtype=float)
    X = np.asarray(X, dtype=float)
    n, k = X.shape
    if w is None:
        wv = np.ones(n)
    else:
        w = np.asarray(w, dtype=float)
        wv = w * n / w.sum() if weight_kind in ("aweight", "pweight") else w.copy()
    if codes:
        D = np.concatenate([np.eye(gq)[c] for c, gq in zip(codes, g)], axis=1)
    else:
        D = np.ones((n, 1))
    Z = np.column_stack([X, D])
    A = np.linalg.pinv(Z.T @ (wv[:, None] * Z), rcond=1e-12)
    beta = A @ (Z.T @ (wv * y))
    e = y - Z @ beta
    h = wv * np.einsum("ij,jk,ik->i", Z, A, Z)
    s = e * wv
    tau = wv if weight_kind == "fweight" else np.ones(n)
    d = tau - h
    ok = d > np.sqrt(np.finfo(float).eps) * tau
    mult = np.zeros(n)
    mult[ok] = (tau[ok] * s[ok] ** 2 / d[ok] ** 2) if hc3 else (s[ok] ** 2 / d[ok])
    # the variance of [X, _cons]: regress on [X, 1] with the FE projected out of X only through
    # the same full-design sandwich, then read off X's block and the constant's combination
    meat = Z.T @ (mult[:, None] * Z)
    Vz = A @ meat @ A
    # the reported constant: mean(y) - mean(X) b, a linear map of the full coefficients
    xbar = (wv @ X) / wv.sum()
    if codes:
        dbar = (wv @ D) / wv.sum()
        L = np.zeros((k + 1, Z.shape[1]))
        L[:k, :k] = np.eye(k)
        L[k, k:] = dbar
        b = L @ beta
    else:
        L = np.eye(k + 1)
        b = beta
    return b, L @ Vz @ L.T, xbar
