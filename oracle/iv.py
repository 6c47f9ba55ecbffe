"""TEST INFRASTRUCTURE — CPU restatement of the reference's IV / 2SLS algebra (numpy).

Only tests/ and bench.py's CPU legs use this module, as the checker; the product (fereg_b200)
never imports it.

The reference (crates/fereg-core/src/iv.rs) runs ivreg2 on the FE-residualized block
[y, exog, endog, inst] with `small` and `noconstant` forced and sdofminus = max(df_a, 1)
(iv.rs:1-16, 376-381). With X = [endog, exog] and Z = [inst, exog] (iv.rs:498-503) and every
cross product weighted by w_v (aw / pw: w n / sum w; fw: w; none: 1):
    b = (X'P_Z X)^-1 X'Z (Z'Z)^-1 Z'y                                   (iv.rs:544-553)
    unadjusted V = rss / (N - K - sdof) (X'P_Z X)^-1                      (iv.rs:613-618)
    robust / cluster V = B S B' * small_adj, B = (X'P_Z X)^-1 X'Z (Z'Z)^-1  (iv.rs:620-633)
with the reghdfe robust multiplier (e^2, e^2 w for fw, (e w_v)^2 for aw / pw), cluster scores
sum_g e w_v z (multiway by inclusion-exclusion), small_adj N / (N - K - sdof) (robust) or
(N - 1) / (N - K - sdof) G / (G - 1) (cluster, G the smallest dimension). pweights imply
robust (ols.rs effective_vce).
"""

import numpy as np

from oracle import oracle


def residualize(codes, g, block, w=None, tol=1e-14, maxiter=100000):
    """The block (original row order) residualized on the FE by the oracle's absorber,
    weighted by the raw weights w."""
    ab = oracle.Absorber(codes, g, w)
    pi = ab.row_order()
    z = np.ascontiguousarray(block[pi])
    ab.residualize(z, tol=tol, maxiter=maxiter)
    res = np.empty_like(block)
    res[pi] = z
    return res


def intersect(a, b):
    key = a.astype(np.int64) * (int(b.max()) + 1) + b.astype(np.int64)
    return np.unique(key, return_inverse=True)[1]


def tsls(Yt, nx, ne, ni, w=None, kind=None, vce="unadjusted", clusters=(), df_a=0):
    """2SLS on the residualized block Yt = [y, exog (nx), endog (ne), inst (ni)] (no
    collinearity handling). Returns b, V in the order [endog, exog], rss and N."""
    n = Yt.shape[0]
    if kind == "pweight" and vce == "unadjusted":
        vce = "robust"
    if w is None:
        wv, big_n = np.ones(n), float(n)
    elif kind == "fweight":
        wv, big_n = w, float(w.sum())
    else:
        wv, big_n = w * n / w.sum(), float(n)
    xc = [1 + nx + j for j in range(ne)] + [1 + j for j in range(nx)]
    zc = [1 + nx + ne + j for j in range(ni)] + [1 + j for j in range(nx)]
    G = Yt.T @ (wv[:, None] * Yt)
    XZ, ZZ, Zy = G[np.ix_(xc, zc)], G[np.ix_(zc, zc)], G[zc, 0]
    ZZi = np.linalg.inv(ZZ)
    XPZXi = np.linalg.inv(XZ @ ZZi @ XZ.T)
    B = XPZXi @ XZ @ ZZi
    beta = B @ Zy
    e = Yt[:, 0] - Yt[:, xc] @ beta
    rss = float(np.sum(wv * e * e))
    k = len(xc)
    sdof = max(df_a, 1)
    nk = big_n - k - sdof
    Z = Yt[:, zc]
    if vce == "unadjusted":
        V = XPZXi * rss / nk
    elif vce == "robust":
        if w is None:
            m = e * e
        elif kind == "fweight":
            m = e * e * w
        else:
            m = (e * wv) ** 2
        V = B @ (Z.T @ (m[:, None] * Z)) @ B.T * big_n / nk
    else:
        sc = (e * wv)[:, None] * Z
        if len(clusters) == 1:
            parts = [(clusters[0], 1.0)]
        else:
            parts = [(clusters[0], 1.0), (clusters[1], 1.0), (intersect(clusters[0], clusters[1]), -1.0)]
        S = np.zeros((len(zc), len(zc)))
        for codes, sign in parts:
            Sg = np.zeros((int(codes.max()) + 1, len(zc)))
            np.add.at(Sg, codes, sc)
            S += sign * Sg.T @ Sg
        gmin = min(int(c.max()) + 1 for c in clusters)
        V = B @ S @ B.T * (big_n - 1) / (big_n - k - sdof) * gmin / (gmin - 1)
    return beta, 0.5 * (V + V.T), rss, big_n
