"""The device WCR11 wild cluster bootstrap (fereg_session_wildboot) against a brute-force refit.

The brute force follows the reference's own oracle of the bootstrap
(crates/fereg-core/tests/wildboot.rs:538 oracle_ols_cluster): explicit FE dummies, the
restricted fit under H0, every draw y*_b = yhat_r + v_{g,b} e_r refitted by weighted least
squares, CRV1 variance per draw, t*_b = (b*_b - b_r) / se*_b. The draws are the reference's
Rademacher signs (SplitMix64 stream (seed, b), bits LSB first: weights.rs:65-79), taken from
the oracle's SplitMix64; full enumeration when 2^G <= reps (weights.rs:39-63). The p-value is
the share of |t*| > |t| + 1e-12 (1 + |t|) (wildboot/mod.rs:529).

Tolerances: t and t* 1e-7 relative (the draws are residualized at tol 1e-12), p-value exact.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import oracle

pytestmark = pytest.mark.gpu


def draws(G, B, seed):
    if G <= 20 and (1 << G) <= B:
        B = 1 << G
        return np.array([[-1.0 if (b >> g) & 1 else 1.0 for g in range(G)] for b in range(B)]), True
    nw = (G + 63) // 64
    V = np.empty((B, G))
    for b in range(B):
        words = oracle.splitmix(seed, nw, index=b)
        for g in range(G):
            V[b, g] = -1.0 if (int(words[g // 64]) >> (g % 64)) & 1 else 1.0
    return V, False


def brute_wcr11(terms, y, X, w, cl, j, r0, V):
    n = len(y)
    W = np.ones(n) if w is None else w
    D = np.concatenate([np.eye(g)[c] for c, g in terms], axis=1)
    sw = np.sqrt(W)[:, None]

    def M(Z):
        coef, *_ = np.linalg.lstsq(D * sw, Z * sw, rcond=None)
        return Z - D @ coef

    Xt = M(X)
    yt = M(y[:, None])[:, 0]
    A = np.linalg.inv(Xt.T @ (W[:, None] * Xt))
    bu = A @ (Xt.T @ (W * yt))
    eu = yt - Xt @ bu
    br = bu - A[:, j] * (bu[j] - r0) / A[j, j]
    er = yt - Xt @ br
    yhat = y - er
    k = X.shape[1]
    G = int(cl.max()) + 1
    df_a = np.linalg.matrix_rank(D)
    ssc = (n - 1) / (n - k - df_a) * G / (G - 1)

    def crv1_jj(E):  # E: n x B residual columns -> V_jj per column
        a = A[j]
        c = Xt @ a
        S = np.zeros((G, E.shape[1]))
        np.add.at(S, cl, (W * c)[:, None] * E)
        return ssc * np.sum(S * S, axis=0)

    se = np.sqrt(crv1_jj(eu[:, None])[0])
    stat = (bu[j] - r0) / se
    Yb = yhat[:, None] + V[:, cl].T * er[:, None]
    Ytb = M(Yb)
    Bb = A @ (Xt.T @ (W[:, None] * Ytb))
    Eb = Ytb - Xt @ Bb
    tb = (Bb[j] - br[j]) / np.sqrt(crv1_jj(Eb))
    eps = 1e-12 * (1 + abs(stat))
    p = np.mean(np.abs(tb) > abs(stat) + eps)
    return stat, se, bu[j], tb, p


def panel(seed, n_ind, years, G, weighted):
    rng = np.random.default_rng(seed)
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    cl = rng.integers(0, G, n).astype(np.uint32)
    _, cl = np.unique(cl, return_inverse=True)
    cl = cl.astype(np.uint32)
    X = rng.standard_normal((n, 3))
    y = 0.0 * X[:, 0] + 0.5 * X[:, 1] - 0.2 * X[:, 2] + rng.standard_normal(n_ind)[ind] + rng.standard_normal(n)
    w = rng.uniform(0.5, 2.0, n) if weighted else None
    return [(ind, n_ind), (year, years)], y, X, w, (cl, int(cl.max()) + 1)


CASES = {
    "random_draws": dict(seed=1, n_ind=60, years=8, G=25, weighted=False, reps=199, tile=64, r0=0.0, coef=0),
    "weighted_nonzero_null": dict(seed=2, n_ind=50, years=6, G=30, weighted=True, reps=99, tile=256, r0=0.3, coef=1),
    "full_enumeration": dict(seed=3, n_ind=40, years=10, G=8, weighted=False, reps=999, tile=100, r0=0.0, coef=0),
}


@pytest.mark.parametrize("case", list(CASES))
def test_wildboot_matches_brute_force(case):
    c = CASES[case]
    terms, y, X, w, (cl, G) = panel(c["seed"], c["n_ind"], c["years"], c["G"], c["weighted"])
    sess = fb.Session([t for t, _ in terms], [g for _, g in terms], [cl], [G], w, "aweight" if w is not None else None)
    pi = sess.row_order()
    rows = np.ascontiguousarray(np.column_stack([y, X])[pi])
    res = sess.wildboot(rows, coef=c["coef"], r0=c["r0"], reps=c["reps"], seed=7, tile=c["tile"], tol=1e-12,
                        maxiter=100000)
    V, full = draws(G, c["reps"], 7)
    wn = None if w is None else w * len(w) / w.sum()  # aweights normalized to sum n (ols.rs:77-108)
    stat, se, point, tb, p = brute_wcr11(terms, y, X, wn, cl, c["coef"], c["r0"], V)
    assert res["full_enum"] == full and res["reps"] == len(tb)
    assert abs(res["point"] - point) <= 1e-9 * max(1.0, abs(point))
    assert abs(res["se"] - se) <= 1e-8 * se
    assert abs(res["stat"] - stat) <= 1e-8 * max(1.0, abs(stat))
    err = np.max(np.abs(res["t_boot"] - tb) / np.maximum(1.0, np.abs(tb)))
    assert err <= 1e-7, err
    assert res["pvalue"] == p


def test_wildboot_fp32_refined_draws():
    """FP32-refined solves of the draws (FP64 statistics) reproduce the FP64 draws' t* to 1e-6."""
    c = CASES["random_draws"]
    terms, y, X, w, (cl, G) = panel(c["seed"], c["n_ind"], c["years"], c["G"], c["weighted"])
    sess = fb.Session([t for t, _ in terms], [g for _, g in terms], [cl], [G])
    rows = np.ascontiguousarray(np.column_stack([y, X])[sess.row_order()])
    a = sess.wildboot(rows, reps=199, seed=7, tile=64, tol=1e-12, maxiter=100000)
    b = sess.wildboot(rows, reps=199, seed=7, tile=64, tol=1e-12, maxiter=100000, boot_tol=1e-10,
                      boot_precision=fb.PREC_F32_REFINED)
    assert np.max(np.abs(a["t_boot"] - b["t_boot"]) / np.maximum(1.0, np.abs(a["t_boot"]))) <= 1e-6
