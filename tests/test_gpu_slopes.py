"""The heterogeneous-slope absorber on the device (slopes.rs SlopeSolver, built by
fereg_absorber_create_terms as solve.rs:338 `build` chooses it) against the dense explicit-dummy
oracle (oracle/slopes.py; the reference checks its SlopeSolver the same way,
crates/fereg-core/tests/slopes.rs:1-120), and the OLS with a slope term against reghdfe
(ols_s16_slopes, tests/ols.rs:827).

Panels follow the reference's test panel (tests/slopes.rs:28-44): indiv x year, firm random or a
band on a ring, a slope x constant within every 7th indiv (degenerate levels) and a slope z; terms
with and without intercepts, weighted and not. Checked: the residualized columns (relative 1e-8
of the column scale at tol 1e-12), the FE fit from the coefficients (fit_rows = column minus
residual), and the kernels one by one (S P, the block-Jacobi preconditioner and the right-hand
side with its statistics, 1e-11) against dense numpy forms of the same operators.
"""

import zlib

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import slopes as osl
from tests._fixtures import load_data, nums
from tests.test_oracle_fixtures import close
from tests.test_oracle_slopes import load_slope_fixtures, prepare_slopes

pytestmark = pytest.mark.gpu


def panel(nindiv, nyear, nfirm, band, seed):
    rng = np.random.default_rng(seed)
    n = nindiv * nyear
    i = np.arange(n)
    indiv = (i // nyear).astype(np.uint32)
    year = (i % nyear).astype(np.uint32)
    if band:
        firm = ((i // nyear * nfirm // nindiv + i % 3) % nfirm).astype(np.uint32)
    else:
        firm = rng.integers(0, nfirm, n).astype(np.uint32)
    x = np.where((i // nyear) % 7 == 0, 1.5, 2.0 + rng.normal(size=n))
    z = rng.normal(size=n)
    w = 0.5 + rng.random(n)
    return dict(indiv=indiv, year=year, firm=firm, x=x, z=z, w=w, n=n), rng


# (factor, intercept, slopes) per term
DESIGNS = {
    "icpt_plus_slope": [("indiv", True, []), ("firm", True, ["x"])],
    "e_with_slope": [("indiv", True, ["x"]), ("year", True, [])],
    "no_intercept": [("indiv", True, []), ("firm", False, ["x", "z"])],
    "three_terms": [("indiv", True, []), ("firm", True, ["z"]), ("year", True, [])],
    "slopes_only": [("firm", False, ["x"]), ("indiv", True, ["z"])],
}
CASES = [(d, band, wtd) for d in DESIGNS for band in (False, True) for wtd in (False, True)]


def build(pan, terms, weighted):
    codes = [pan[f] for f, _, _ in terms]
    g = [int(c.max()) + 1 for c in codes]
    icpt = [i for _, i, _ in terms]
    sl = [[pan[s] for s in ss] for _, _, ss in terms]
    w = pan["w"] if weighted else None
    return codes, g, icpt, sl, w


@pytest.mark.parametrize("design,band,weighted", CASES, ids=[f"{d}-{'band' if b else 'rand'}-{'w' if w else 'u'}"
                                                          for d, b, w in CASES])
def test_slope_residualize_matches_dense(design, band, weighted):
    pan, rng = panel(80, 6, 15, band, seed=zlib.crc32(f"{design}-{band}-{weighted}".encode()))
    codes, g, icpt, sl, w = build(pan, DESIGNS[design], weighted)
    ab = fb.Absorber(codes, g, w, intercept=icpt, slopes=sl)
    assert ab.has_slopes
    n = pan["n"]
    Z = np.column_stack([rng.normal(size=n) + 5 + 3 * pan["x"], rng.normal(size=n), pan["x"] * pan["z"]])
    want = osl.residualize(codes, g, icpt, sl, Z, w)
    pi = ab.row_order()
    rows = np.ascontiguousarray(Z[pi])
    res = ab.residualize(rows, tol=1e-12, maxiter=100000, want_coefs=True)
    got = np.empty_like(rows)
    got[pi] = rows
    scale = np.abs(Z).max(axis=0)
    assert np.abs(got - want).max(axis=0).max() <= 1e-8 * scale.max(), np.abs(got - want).max(axis=0)
    # the FE fit from the coefficients
    for col in range(Z.shape[1]):
        fit = ab.fit_rows(res["coefs"], col)
        assert np.abs(fit - (Z[pi, col] - rows[:, col])).max() <= 1e-8 * scale[col]
    tv = ab.term_values(res["coefs"], 0)
    assert sum(len(v) for v in tv) == ab.term_values_len


def dense_operators(ab, codes, g, icpt, sl, w):
    """S, its right-hand side map and the block-Jacobi preconditioner densely, in the solver's
    coordinate order (small blocks first, levels in order, slots intercept then slopes)."""
    st = ab.slope_structure()
    e = st["e"]
    n = len(codes[0])
    wv = np.ones(n) if w is None else np.asarray(w)
    DE = osl.design([codes[e]], [g[e]], [icpt[e]], [sl[e]])
    cols = []
    for q in st["block_terms"]:
        dm = np.eye(g[q])[codes[q]]
        slot = ([np.ones(n)] if icpt[q] else []) + list(sl[q])
        b = len(slot)
        blk = np.zeros((n, g[q] * b))
        for d, v in enumerate(slot):
            blk[:, d::b] = dm * v[:, None]
        cols.append(blk)
    DB = np.concatenate(cols, axis=1)
    M = DE.T @ (wv[:, None] * DE)
    Pm = DE @ np.linalg.pinv(M, rcond=1e-12) @ (DE.T * wv)  # the weighted projection on E
    resid = np.eye(n) - Pm
    S = DB.T @ (wv[:, None] * (resid @ DB))
    Rhs = DB.T @ (wv[:, None] * resid)
    return st, S, Rhs, resid


@pytest.mark.parametrize("design", list(DESIGNS))
@pytest.mark.parametrize("weighted", [False, True])
def test_slope_kernels_match_dense(design, weighted):
    pan, rng = panel(30, 5, 8, False, seed=11)
    codes, g, icpt, sl, w = build(pan, DESIGNS[design], weighted)
    ab = fb.Absorber(codes, g, w, intercept=icpt, slopes=sl)
    pi = ab.row_order()
    # the operators on the row order
    codes_r = [c[pi] for c in codes]
    sl_r = [[x[pi] for x in t] for t in sl]
    w_r = None if w is None else w[pi]
    st, S, Rhs, resid = dense_operators(ab, codes_r, g, icpt, sl_r, w_r)
    m = st["m"]
    P = rng.normal(size=(m, 3))
    got = ab.slope_apply(P)
    assert np.abs(got - S @ P).max() <= 1e-11 * max(1.0, np.abs(S @ P).max())
    V = rng.normal(size=(len(pi), 3))
    y, stats = ab.slope_rhs(V)
    assert np.abs(y - Rhs @ V).max() <= 1e-11 * max(1.0, np.abs(Rhs @ V).max())
    wv = np.ones(len(pi)) if w_r is None else w_r
    E = resid @ V
    assert np.allclose(stats[0], (wv[:, None] * V * V).sum(0), rtol=1e-12)
    assert np.allclose(stats[1], (wv[:, None] * V).sum(0), rtol=1e-12)
    assert np.allclose(stats[2], (wv[:, None] * E * E).sum(0), rtol=1e-10)
    # block Jacobi: the b x b diagonal blocks of S, redundant slots dropped
    blocks = []
    for q in st["block_terms"]:
        b = int(icpt[q]) + len(sl[q])
        blocks += [b] * g[q]
    jlen = sum(b * b for b in blocks)
    ws = ab.slope_weight_state(jlen)
    Rr = rng.normal(size=(m, 2))
    z = ab.slope_precond(Rr)
    zw = np.zeros_like(Rr)
    c0 = jo = 0
    for b in blocks:
        Jb = ws["jinv"][jo:jo + b * b].reshape(b, b)
        zw[c0:c0 + b] = Jb @ Rr[c0:c0 + b]
        # the inverse is the generalized inverse of the diagonal block on its kept slots
        keep = ~ws["redundant"][c0:c0 + b]
        Sb = S[c0:c0 + b, c0:c0 + b][np.ix_(keep, keep)]
        if keep.any() and np.linalg.matrix_rank(Sb) == keep.sum():
            assert np.allclose(Jb[np.ix_(keep, keep)] @ Sb, np.eye(keep.sum()), atol=1e-8)
        c0 += b
        jo += b * b
    assert np.abs(z - zw).max() <= 1e-12 * max(1.0, np.abs(zw).max())


def test_session_ols_with_slopes_matches_reghdfe_s16():
    data = load_data()
    fix = load_slope_fixtures()[0]
    spec = fix["spec"]
    alive, nsing, terms, slopes = prepare_slopes(spec, data)
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms], num_singletons=nsing,
                      intercept=spec["intercept"], slopes=slopes)
    pi = sess.row_order()
    cols = [data[spec["y"]][alive]] + [data[x][alive] for x in spec["x"]]
    rows = np.ascontiguousarray(np.stack(cols, axis=1)[pi])
    res = sess.ols(rows, vce="unadjusted", tol=1e-14, maxiter=100000)
    assert close(res["b"], nums(fix["b"]), 1e-7), (res["b"], fix["b"])
    assert close(res["V"].ravel(), nums(fix["V"]), 1e-6)
    assert np.array_equal(res["dof_table"].ravel(), nums(fix["dof_table"]))
    sc = res["scalars"]
    for k in ("N", "df_a", "df_r", "num_singletons"):
        assert sc[k] == fix["scalars"][k], k
    assert abs(sc["rss"] - fix["scalars"]["rss"]) <= 1e-6 * fix["scalars"]["rss"]
