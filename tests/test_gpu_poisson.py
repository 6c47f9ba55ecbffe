"""The device Poisson PML (fereg_session_poisson) against a dense explicit-dummy fit.

The Poisson maximum-likelihood estimate is unique, so the reference here is the same model fitted
densely by the oracle (oracle/glm.py): explicit FE dummies, IRLS on the full design until the
deviance stops changing (relative 1e-15). The variance follows ppmlhdfe's conventions as the reference restates them
(crates/fereg-core/src/glm/mod.rs:1-22, 1053-1140): robust
(X~'WX~)^-1 [sum (y - mu)^2 x~ x~'] (X~'WX~)^-1 N / (N - 1), clustered with G / (G - 1), where X~
is X residualized on the dummies with weights mu.

Tolerances: b 1e-7, V 1e-6 relative, deviance and log-likelihood 1e-9 relative.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import glm as oglm

pytestmark = pytest.mark.gpu


def dense_ppml(terms, y, X, cl=None):
    return oglm.dense_glm("poisson", terms, y, X, "robust" if cl is None else "cluster", cl)


def panel(seed, n_ind, years, n_firm, k):
    rng = np.random.default_rng(seed)
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    firm = rng.integers(0, n_firm, n).astype(np.uint32)
    _, firm = np.unique(firm, return_inverse=True)
    firm = firm.astype(np.uint32)
    X = rng.standard_normal((n, k))
    eta = 0.3 * X[:, 0] - 0.2 * X[:, 1] + 0.5 * rng.standard_normal(n_ind)[ind] + 0.3 * rng.standard_normal(years)[year]
    y = rng.poisson(np.exp(eta + 0.5)).astype(float)
    # drop individuals whose counts are all zero (the `fe` separation rule of the preparation)
    keep_ind = np.bincount(ind, weights=y, minlength=n_ind) > 0
    keep = keep_ind[ind]
    _, ind2 = np.unique(ind[keep], return_inverse=True)
    _, firm2 = np.unique(firm[keep], return_inverse=True)
    return (ind2.astype(np.uint32), int(ind2.max()) + 1), (year[keep], years), \
        (firm2.astype(np.uint32), int(firm2.max()) + 1), y[keep], X[keep]


@pytest.mark.parametrize("vce", ["robust", "cluster"])
def test_poisson_matches_dense_fit(vce):
    (ind, gi), (year, gy), (firm, gf), y, X = panel(5, 120, 6, 15, 2)
    terms = [(ind, gi), (year, gy)]
    sess = fb.Session([ind, year], [gi, gy], [firm], [gf])
    pi = sess.row_order()
    rows = np.ascontiguousarray(np.column_stack([y, X])[pi])
    res = sess.poisson(rows, vce=vce, tol=1e-12, inner_maxiter=100000)
    b, V, dev, ll = dense_ppml(terms, y, X, (firm, gf) if vce == "cluster" else None)
    assert res["converged"]
    assert np.max(np.abs(res["b"] - b) / np.maximum(1.0, np.abs(b))) <= 1e-7, (res["b"], b)
    assert np.max(np.abs(res["V"] - V)) <= 1e-6 * np.max(np.abs(V)), (res["V"], V)
    assert abs(res["deviance"] - dev) <= 1e-9 * dev
    assert abs(res["ll"] - ll) <= 1e-9 * abs(ll)


def test_poisson_absorbed_regressor_is_flagged():
    """A regressor constant within each individual is absorbed by the FE (status 2, b = 0)."""
    (ind, gi), (year, gy), (firm, gf), y, X = panel(6, 100, 5, 10, 2)
    xa = np.random.default_rng(1).standard_normal(gi)[ind]
    X3 = np.column_stack([X, xa])
    sess = fb.Session([ind, year], [gi, gy])
    rows = np.ascontiguousarray(np.column_stack([y, X3])[sess.row_order()])
    res = sess.poisson(rows, tol=1e-12, inner_maxiter=100000)
    assert list(res["status"]) == [0, 0, 2] and res["b"][2] == 0.0
    b, V, dev, ll = dense_ppml([(ind, gi), (year, gy)], y, X)
    assert np.max(np.abs(res["b"][:2] - b)) <= 1e-7 * max(1.0, np.max(np.abs(b)))
