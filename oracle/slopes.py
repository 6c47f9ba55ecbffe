"""TEST INFRASTRUCTURE — dense CPU restatement of the reference's heterogeneous-slope absorber
(numpy), the checker of the B200 slope solver.

Only tests/ use this module; the product (fereg_b200) never imports it.

The residualization of slopes.rs (SlopeSolver::residualize, slopes.rs:2338-2433) is the weighted
projection of every column off the span of the FE design: per term the intercept dummies (when the
term has an intercept) and one dummy times each slope variable (`fe#c.x`). The projection is unique,
so the dense restatement builds that design explicitly and solves the weighted least-squares
problem (the reference's own tests check SlopeSolver against the same dense explicit-dummy oracle,
crates/fereg-core/tests/slopes.rs:1-120). The FE fit (Absorber::fit_rows, slopes.rs:1559) is the
column minus its residual.

The degrees of freedom restate dof.rs:64-180 (estimate_dof) with slopes: one slot per intercept,
then one per slope; intercept slots nested in a cluster dimension are fully redundant; every
remaining intercept but the first keeps one redundant level; the first pair of remaining
intercepts adds its mobility groups; a slope is redundant on the levels where it is constant
(term with intercept) or zero (term without) after scaling by its standard deviation
(dof.rs:255-272).

The OLS (ols.rs:263-470) follows reghdfe: b from the residualized block, _cons = weighted mean of
y minus the weighted means of X times b, V from the bordered inverse (vcov.rs:220) times
rss / df_r with df_r = N - df_a - k (iid).
"""

import numpy as np

from oracle import oracle


def design(codes, g, intercept, slopes):
    """The dense FE design: per term its intercept dummies, then one dummy block per slope."""
    cols = []
    for q, (c, gq) in enumerate(zip(codes, g)):
        dummies = np.eye(gq)[np.asarray(c)]
        if intercept[q]:
            cols.append(dummies)
        for x in slopes[q]:
            cols.append(dummies * np.asarray(x)[:, None])
    return np.concatenate(cols, axis=1)


def residualize(codes, g, intercept, slopes, Z, w=None):
    """Columns of Z (n x r, kept order) minus their weighted projection on the FE design."""
    D = design(codes, g, intercept, slopes)
    Z = np.asarray(Z, dtype=float)
    sw = np.ones(len(Z)) if w is None else np.sqrt(np.asarray(w, dtype=float))
    beta, *_ = np.linalg.lstsq(D * sw[:, None], Z * sw[:, None], rcond=1e-13)
    return Z - D @ beta


def redundant_slope_levels(codes, g, x, intercept):
    """dof.rs:255-272."""
    x = np.asarray(x, dtype=float)
    sd = max(np.std(x, ddof=1), 1e-3)
    v = x / sd
    lo = np.full(g, np.inf)
    hi = np.full(g, -np.inf)
    np.minimum.at(lo, codes, v)
    np.maximum.at(hi, codes, v)
    if intercept:
        return int(np.sum(hi - lo <= 1e-6))
    return int(np.sum(np.abs(lo) + np.abs(hi) <= 1e-6))


def estimate_dof(codes, g, intercept, slopes, clusters=()):
    """dof.rs:64-180 with the default options; returns (slots [k, m, exact, nested], df_a)."""
    slots, icpt_term, first_slope = [], [], {}
    for q in range(len(codes)):
        if intercept[q]:
            slots.append([g[q], 0, False, False])
            icpt_term.append(q)
        if slopes[q]:
            first_slope[q] = len(slots)
        for _ in slopes[q]:
            slots.append([g[q], 0, False, False])
            icpt_term.append(None)
    live = [t is not None for t in icpt_term]
    nested = 0
    for cc in clusters:
        if not any(live):
            break
        for i, t in enumerate(icpt_term):
            if not live[i] or slots[i][2]:
                continue
            c = np.asarray(codes[t])
            pairs = np.unique(np.stack([c, np.asarray(cc)], axis=1), axis=0)
            if len(np.unique(pairs[:, 0])) == len(pairs):  # every level in one cluster
                slots[i][1] = slots[i][0]
                slots[i][2] = slots[i][3] = True
                nested += slots[i][0]
                live[i] = False
    remaining = sum(live)
    if remaining > 1 or (remaining > 0 and nested > 0):
        skip = nested == 0
        for i in range(len(slots)):
            if not live[i]:
                continue
            if skip:
                skip = False
                continue
            slots[i][1] = 1
    for i in range(len(slots)):
        if live[i]:
            slots[i][2] = True
            break
    idx = [i for i in range(len(slots)) if live[i]]
    if len(idx) >= 2:
        for a in range(len(idx)):
            for b in range(a + 1, len(idx)):
                ta, tb = icpt_term[idx[a]], icpt_term[idx[b]]
                m = oracle.mobility_groups(codes[ta], g[ta], codes[tb], g[tb])
                slots[idx[b]][1] = max(slots[idx[b]][1], m)
                if a == 0 and b == 1:
                    slots[idx[b]][2] = True
    for q, i0 in first_slope.items():
        for k, x in enumerate(slopes[q]):
            cnt = redundant_slope_levels(codes[q], g[q], x, intercept[q])
            if cnt > 0:
                slots[i0 + k][1] = cnt
    df_a = sum(s[0] for s in slots) - sum(s[1] for s in slots)
    return slots, df_a


def ols_iid(codes, g, intercept, slopes, y, X):
    """OLS of y on X (unweighted, iid) with the slope terms absorbed: b and V of [X..., _cons],
    the dof slots and df_a."""
    Z = np.column_stack([y] + list(X))
    Zr = residualize(codes, g, intercept, slopes, Z)
    yt, Xt = Zr[:, 0], Zr[:, 1:]
    A = np.linalg.inv(Xt.T @ Xt)
    b = A @ Xt.T @ yt
    n, k = Xt.shape
    slots, df_a = estimate_dof(codes, g, intercept, slopes)
    rss = float(np.sum((yt - Xt @ b) ** 2))
    df_r = n - df_a - k
    xbar = Z[:, 1:].mean(axis=0)
    b0 = Z[:, 0].mean() - xbar @ b
    Ax = A @ xbar
    bread = np.zeros((k + 1, k + 1))
    bread[:k, :k] = A
    bread[:k, k] = bread[k, :k] = -Ax
    bread[k, k] = 1.0 / n + xbar @ Ax
    return np.append(b, b0), bread * rss / df_r, slots, df_a
