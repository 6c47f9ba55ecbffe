"""TEST INFRASTRUCTURE — dense CPU restatement of the reference's GLM fits (numpy).

Only tests/ and bench.py's CPU legs use this module, as the checker; the product (fereg_b200)
never imports it.

The Poisson and logit MLEs with absorbed fixed effects are unique, so the dense restatement fits
the same model with explicit FE dummies: IRLS on the full design (glm/irls.rs:367-560 with the
families of glm/family.rs:101-147: Poisson w = mu, z = eta - 1 + y / mu; logit w = mu (1 - mu),
z = eta + (y - mu) / w) until the deviance stops changing (relative 1e-15). The variance follows
glm/mod.rs:1-22: X~ is X residualized on the dummies with the final weights, robust
(X~'WX~)^-1 [sum (y - mu)^2 x~ x~'] (X~'WX~)^-1 N / (N - 1), clustered with G / (G - 1), logit
`oim` the inverse Hessian (X~'WX~)^-1.
"""

import numpy as np
from scipy.special import expit, gammaln


def dense_glm(family, terms, y, X, vce="robust", cl=None, maxiter=200):
    """terms: list of (codes, levels); cl: (codes, G), or a list of them, for vce="cluster". Returns b, V, deviance,
    log-likelihood."""
    n = len(y)
    D = np.concatenate([np.eye(g)[c] for c, g in terms], axis=1)
    Z = np.concatenate([X, D], axis=1)
    if family == "poisson":
        mu = (y + y.mean()) / 2
        eta = np.log(mu)
    else:
        mu = (y + 0.5) / 2
        eta = np.log(mu / (1 - mu))
    dev_old = np.inf
    for _ in range(maxiter):
        if family == "poisson":
            w = mu
            z = eta - 1 + y / mu
        else:
            w = mu * (1 - mu)
            z = eta + (y - mu) / w
        sw = np.sqrt(w)[:, None]
        coef, *_ = np.linalg.lstsq(Z * sw, z * sw[:, 0], rcond=None)
        eta = Z @ coef
        if family == "poisson":
            mu = np.exp(eta)
            dev = 2 * np.sum(np.where(y > 0, y * np.log(np.where(y > 0, y, 1) / mu), 0) - (y - mu))
        else:
            mu = expit(eta)
            dev = -2 * np.sum(y * eta - np.logaddexp(0, eta))
        if abs(dev - dev_old) <= 1e-15 * dev:
            break
        dev_old = dev
    k = X.shape[1]
    b = coef[:k]
    w = mu if family == "poisson" else mu * (1 - mu)
    sw = np.sqrt(w)[:, None]
    cd, *_ = np.linalg.lstsq(D * sw, X * sw, rcond=None)
    Xt = X - D @ cd
    A = np.linalg.inv(Xt.T @ (w[:, None] * Xt))
    s = (y - mu)[:, None] * Xt
    if vce == "oim":
        V = A
    elif vce == "robust":
        V = A @ (s.T @ s) @ A * n / (n - 1)
    else:
        codes, G = cl
        S = np.zeros((G, k))
        np.add.at(S, codes, s)
        V = A @ (S.T @ S) @ A * G / (G - 1)
    if family == "poisson":
        ll = np.sum(y * eta - mu - gammaln(y + 1))
    else:
        ll = np.sum(y * eta - np.logaddexp(0, eta))
    return b, V, dev, ll


def cluster_sandwich(A, s, dims):
    """A (sum over clusters of the score sums' outer products) A with reghdfe's multiway rule
    (vcov.rs:480-560 multiway_meat): inclusion-exclusion over the intersections of the cluster
    dimensions, the G/(G-1) factor of the smallest dimension, and the negative eigenvalues of a
    multiway V clipped to 0. dims: (codes per row, G) in the rows' order."""
    from itertools import combinations

    k = s.shape[1]
    meat = np.zeros((k, k))
    for size in range(1, len(dims) + 1):
        for sub in combinations(dims, size):
            key = np.zeros(len(s), dtype=np.int64)
            for c, G in sub:
                key = key * G + c
            _, inv = np.unique(key, return_inverse=True)
            S = np.zeros((inv.max() + 1, k))
            np.add.at(S, inv, s)
            meat += (-1.0) ** (size + 1) * (S.T @ S)
    gmin = min(G for _, G in dims)
    V = A @ meat @ A * gmin / (gmin - 1)
    if len(dims) > 1:
        lam, Q = np.linalg.eigh(V)
        if lam.min() < 0:
            V = (Q * np.maximum(lam, 0)) @ Q.T
    return V


def _predict_eps(hist, eps):
    """ppmlhdfe predict_eps (glm/irls.rs:105-140): the cubic without a constant through the last
    three (i, ln eps_i), evaluated at i = 4; NaN until three values are known."""
    le = np.log(eps) if eps > 0 else np.nan
    known = [v for v in hist if not np.isnan(v)]
    abort = len(known) + 1 < 3
    if len(known) < 3:
        hist[:] = known + [le]
    else:
        hist[:] = known[1:] + [le]
    if abort or len(hist) < 3 or any(np.isnan(v) for v in hist):
        return np.nan
    A = np.array([[1.0, 1.0, 1.0], [2.0, 4.0, 8.0], [3.0, 9.0, 27.0]])
    c = np.linalg.solve(A, np.array(hist))
    return float(np.exp(4 * c[0] + 16 * c[1] + 64 * c[2]))


def irls_absorbed(codes, g, y, X, family, vce="robust", cl=None, tol=1e-8, itol=1e-10, maxiter=1000, state=None):
    """IRLS with the fixed effects absorbed by the oracle's FE solver (the reference's loop,
    glm/irls.rs:367-560): each iteration sets the family's weights on the absorber, residualizes
    [z, X] warm-started from the previous FE coefficients, fits the weighted regression on the
    residualized block, and updates eta = z - e; the inner tolerance starts at max(1e-4, tol)
    and is tightened 10x when the deviance change falls below it, down to
    max(1e-12, min(itol, 0.1 tol)) (glm/mod.rs:826);
    convergence when the relative deviance change is below tol at the tightest inner tolerance.
    A regressor that the fixed effects absorb (after the first iteration's solve, weighted
    residual sum of squares <= min(1e-6, tol / 10) times its raw sum of squares, the stage-1 rule
    of ols.rs:38) keeps being residualized but leaves the fit: its coefficient and its row and
    column of V are 0. Unweighted samples, no separation checks. Returns b, V, deviance,
    log-likelihood, iterations."""
    from oracle import oracle

    ab = oracle.Absorber(codes, g)
    pi = ab.row_order()
    y = np.asarray(y, dtype=np.float64)[pi]
    X = np.asarray(X, dtype=np.float64)[pi]
    n, k = X.shape
    if family == "poisson":
        mu = (y + y.mean()) / 2
        eta = np.log(mu)
    else:
        mu = (y + 0.5) / 2
        eta = np.log(mu / (1 - mu))
    highest = max(1e-12, min(itol, 0.1 * tol))
    tol_in = max(1e-4, tol)
    dev_old = np.nan
    warm = None
    eps, alt_tol, hist = np.nan, np.inf, []
    sumsq = np.sum(X * X, axis=0)
    keep = np.arange(k)
    for it in range(1, maxiter + 1):
        predicted = _predict_eps(hist, eps)
        if family == "poisson":
            w = mu
            z = eta - 1 + y / mu
        else:
            w = mu * (1 - mu)
            z = eta + (y - mu) / w
        ab.set_weights(w)
        B = np.ascontiguousarray(np.column_stack([z, X]))
        out = ab.residualize(B, tol=tol_in, maxiter=100000, want_coefs=True, warm=warm)
        warm = out["coefs"]
        if it == 1:
            ss = np.sum(w[:, None] * B[:, 1:] ** 2, axis=0)
            keep0 = np.flatnonzero(ss > min(1e-6, tol / 10) * sumsq)
            # then the columns collinear with earlier kept ones (the sweep's pivot order)
            sw = np.sqrt(w)
            kk = []
            for j in keep0:
                M = B[:, [1 + q for q in kk + [j]]] * sw[:, None]
                if np.linalg.matrix_rank(M, tol=1e-9 * np.linalg.norm(M)) == len(kk) + 1:
                    kk.append(j)
            keep = np.array(kk, dtype=int)
        Xt, zt = B[:, 1 + keep], B[:, 0]
        A = np.linalg.inv(Xt.T @ (w[:, None] * Xt))
        b = A @ (Xt.T @ (w * zt))
        e = zt - Xt @ b
        eta = z - e
        if family == "poisson":
            mu = np.maximum(np.exp(eta), 100 * np.finfo(float).eps)
            dev = 2 * np.sum(np.where(y > 0, y * (np.log(np.where(y > 0, y, 1)) - eta), 0) + (mu - y))
        else:
            mu = np.clip(expit(eta), 100 * np.finfo(float).eps, 1 - 100 * np.finfo(float).eps)
            dev = 2 * np.sum(np.logaddexp(0, eta) - y * eta)
        if it > 1:
            delta = dev_old - dev
            if dev < 0.1 * delta:
                delta = dev
            eps = abs(delta) / max(min(dev, dev_old), 0.1)
            if eps < tol and tol_in <= 1.1 * highest:
                break
            # irls.rs:900-911: a decade, or down to the decade of 0.1 eps of the previous
            # tightening, and one more when the predicted eps is below tol
            if eps < tol_in:
                tol_in = max(min(0.1 * tol_in, alt_tol), highest)
                alt_tol = 10.0 ** (-np.ceil(np.log10(1.0 / max(0.1 * eps, np.finfo(float).eps))))
            if not np.isnan(predicted) and tol <= predicted <= eps and 1.1 <= tol_in / highest <= 10.1:
                tol_in *= 0.1
        dev_old = dev
    s = (e * w)[:, None] * Xt
    if state is not None:  # the final iteration's quantities, in row order
        state.update(w=w, e=e, Xt=Xt, X=X[:, keep], A=A, pi=pi, keep=keep)
    if vce == "oim":
        Vk = A
    elif vce == "robust":
        Vk = A @ (s.T @ s) @ A * n / (n - 1)
    else:
        Vk = cluster_sandwich(A, s, [(np.asarray(c)[pi], G) for c, G in (cl if isinstance(cl, list) else [cl])])
    if family == "poisson":
        ll = np.sum(y * eta - mu - gammaln(y + 1))
    else:
        ll = np.sum(y * eta - np.logaddexp(0, eta))
    bf = np.zeros(k)
    bf[keep] = b
    V = np.zeros((k, k))
    V[np.ix_(keep, keep)] = Vk
    return bf, V, dev, ll, it


def relu_separation(codes, g, y, X, itol=1e-10):
    """ReLU separation check (glm/separation.rs:61-196, ppmlhdfe 2.3.3 relu_fix_separation) on
    the dense FE design: the method of weighting (M = ceil(eps^-1/2) on y > 0, 1 on y = 0) of the
    working variable u (start 1[y = 0]) regressed on X / sd (unweighted sd floored at 1e-3,
    glm/mod.rs:4-6) and the FE dummies; regressors absorbed by the FE (sum x~^2 / sum x^2 <=
    min(1e-6, itol / 10)) or collinear with the others on the first solve leave the regression.
    Each step: xbd = u - e, 0 off the boundary and within [-0.1 delta, delta] with delta =
    max(u'u / M ratio^2, 1e-8) + 1e-4 (ratio: norm(X, 1) of the y > 0 rows over the y = 0 rows);
    stop when xbd >= 0 on the boundary, or when no boundary residual (0 within 1e-8) is negative
    (then rows with residual > delta leave); else u = max(xbd, 0) on the boundary. Past 100
    steps it continues while the negative predictions fall by 1% over 10 steps (at most 2000).
    Returns the separated rows (bool) and whether the check certified its result."""
    y = np.asarray(y, dtype=float)
    X = np.asarray(X, dtype=float).reshape(len(y), -1)
    n, k = X.shape
    bd = y == 0
    if not bd.any():
        return np.zeros(n, dtype=bool), True
    D = np.concatenate([np.eye(gq)[c] for c, gq in zip(codes, g)], axis=1) if codes else np.ones((n, 1))
    sd = np.maximum(X.std(axis=0, ddof=1), 1e-3) if k else np.ones(0)
    Xs = X / sd if k else X
    big_m = np.ceil(np.finfo(float).eps ** -0.5)
    w = np.where(bd, 1.0, big_m)
    sw = np.sqrt(w)
    if k:
        a = np.abs(Xs[~bd]).sum(axis=0).max() if (~bd).any() else 0.0
        c = np.abs(Xs[bd]).sum(axis=0).max()
        with np.errstate(divide="ignore", invalid="ignore"):
            ratio = a / c
        ratio = max(ratio, 1.0) if np.isfinite(ratio) else 1.0
    else:
        ratio = 1.0

    def resid_on_d(B):
        beta, *_ = np.linalg.lstsq(D * sw[:, None], B * sw[:, None], rcond=None)
        return B - D @ beta

    u = bd.astype(float)
    keep = None
    hist = []
    it = 0
    while True:
        it += 1
        B = np.column_stack([u, Xs])
        Bt = resid_on_d(B)
        if keep is None:
            keep = []
            if k:
                ss = (w[:, None] * Bt[:, 1:] ** 2).sum(axis=0)
                raw = (Xs ** 2).sum(axis=0)
                cand = [j for j in range(k) if raw[j] > 0 and not ss[j] / raw[j] <= min(1e-6, itol / 10)]
                for j in cand:  # sequential rank test (the sweep's pivot order)
                    M = Bt[:, [1 + q for q in keep + [j]]] * sw[:, None]
                    if np.linalg.matrix_rank(M, tol=1e-9 * np.linalg.norm(M)) == len(keep) + 1:
                        keep.append(j)
        if keep:
            Xt = Bt[:, [1 + q for q in keep]]
            b, *_ = np.linalg.lstsq(Xt * sw[:, None], Bt[:, 0] * sw, rcond=None)
            e = Bt[:, 0] - Xt @ b
        else:
            e = Bt[:, 0].copy()
        uu = float(u @ u)
        delta = max(uu / big_m * ratio * ratio, 1e-8) + 1e-4
        xbd = u - e
        xbd[~bd | ((-0.1 * delta <= xbd) & (xbd <= delta))] = 0.0
        if np.all(xbd[bd] >= 0):
            return bd & (xbd > 0), True
        e[np.abs(e) <= 1e-8] = 0.0
        if e[bd].min() >= 0:
            xbd[bd & (e > delta)] = 0.0
            return bd & (xbd > 0), True
        hist.append(float(-xbd[bd & (xbd < 0)].sum()))
        stalled = len(hist) > 10 and hist[-1] > 0.99 * hist[-11]
        if it >= 100 and (stalled or it >= 2000):
            return np.zeros(n, dtype=bool), False
        u[bd] = np.maximum(xbd[bd], 0.0)
