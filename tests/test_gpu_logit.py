"""The device logit (fereg_session_glm, logit family) against Stata logit fixtures and the oracle.

Stata `logit y x1 x2 i.fe1 i.fe2` (tests/glm.rs:659-672 of the reference, here with the dummies
absorbed): the slopes' b and V (oim, robust, cluster) and the log-likelihood, tolerances of the
reference's harness (b 1e-7, V 1e-6, ll 1e-7). A larger synthetic panel is checked against the
oracle's dense logit (oracle/glm.py) at the same tolerances.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import glm as oglm
from oracle import oracle
from tests._fixtures import load_csv, load_json

pytestmark = pytest.mark.gpu

DATA = load_csv("glm_logit.csv")
FIXTURES = load_json("logit_fixtures.json")


@pytest.mark.parametrize("fix", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_logit_matches_stata(fix):
    spec = fix["spec"]
    terms = [oracle.factorize(DATA[f]) for f in spec["absorb"]]
    alive, nsing = oracle.drop_singletons([c for c, _ in terms], [g for _, g in terms])
    assert alive.all() and nsing == 0 and all(s == 1 for s in fix["sample"])
    cl = [oracle.factorize(DATA[spec["cluster"]])] if spec["cluster"] else []
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms], [c for c, _ in cl], [g for _, g in cl])
    rows = np.ascontiguousarray(np.column_stack([DATA["y"], DATA["x1"], DATA["x2"]])[sess.row_order()])
    res = sess.logit(rows, vce=spec["vce"], tol=1e-12, inner_maxiter=100000)
    assert res["converged"] and not res["status"].any()
    bw = np.array(fix["b"])
    Vw = np.array(fix["V"]).reshape(2, 2)
    assert np.max(np.abs(res["b"] - bw) / np.abs(bw)) <= 1e-7, (res["b"], bw)
    assert np.max(np.abs(res["V"] - Vw)) <= 1e-6 * np.max(np.abs(Vw)), (res["V"], Vw)
    ll = fix["scalars"]["ll"]
    assert abs(res["ll"] - ll) <= 1e-7 * abs(ll)
    assert abs(res["deviance"] + 2 * ll) <= 1e-7 * abs(ll)


def panel(seed, n_ind, years, k):
    rng = np.random.default_rng(seed)
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    X = rng.standard_normal((n, k))
    eta = 0.6 * X[:, 0] - 0.4 * X[:, 1] + 0.7 * rng.standard_normal(n_ind)[ind] + 0.3 * rng.standard_normal(years)[year]
    y = (rng.random(n) < 1 / (1 + np.exp(-eta))).astype(float)
    # the `fe` separation rule: drop individuals whose outcomes never vary
    s = np.bincount(ind, weights=y, minlength=n_ind)
    keep = ((s > 0) & (s < years))[ind]
    _, ind2 = np.unique(ind[keep], return_inverse=True)
    return (ind2.astype(np.uint32), int(ind2.max()) + 1), (year[keep], years), y[keep], X[keep]


@pytest.mark.parametrize("vce", ["oim", "robust"])
def test_device_logit_matches_dense_oracle(vce):
    (ind, gi), (year, gy), y, X = panel(21, 300, 8, 3)
    sess = fb.Session([ind, year], [gi, gy])
    rows = np.ascontiguousarray(np.column_stack([y, X])[sess.row_order()])
    res = sess.logit(rows, vce=vce, tol=1e-12, inner_maxiter=100000)
    b, V, dev, ll = oglm.dense_glm("logit", [(ind, gi), (year, gy)], y, X, vce)
    assert np.max(np.abs(res["b"] - b) / np.maximum(1.0, np.abs(b))) <= 1e-7
    assert np.max(np.abs(res["V"] - V)) <= 1e-6 * np.max(np.abs(V))
    assert abs(res["ll"] - ll) <= 1e-9 * abs(ll)


def test_device_logit_rejects_non_binary_outcome():
    (ind, gi), (year, gy), y, X = panel(22, 50, 5, 2)
    sess = fb.Session([ind, year], [gi, gy])
    rows = np.ascontiguousarray(np.column_stack([y, X])[sess.row_order()])
    rows[0, 0] = 2.0
    with pytest.raises(fb.FeregError) as e:
        sess.logit(rows)
    assert e.value.rc == 198
