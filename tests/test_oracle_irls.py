"""The oracle's absorbed IRLS (oracle/glm.py irls_absorbed, over the oracle's FE solver) agrees
with its dense explicit-dummy fit and with the Stata logit fixtures: b 1e-7, V 1e-6, ll 1e-9."""

import numpy as np
import pytest

from oracle import glm as oglm
from oracle import oracle
from tests._fixtures import load_csv, load_json


def panel(seed, n_ind, years, family):
    rng = np.random.default_rng(seed)
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    X = rng.standard_normal((n, 2))
    eta = 0.4 * X[:, 0] - 0.3 * X[:, 1] + 0.5 * rng.standard_normal(n_ind)[ind]
    if family == "poisson":
        y = rng.poisson(np.exp(eta + 0.3)).astype(float)
        keep = (np.bincount(ind, weights=y, minlength=n_ind) > 0)[ind]
    else:
        y = (rng.random(n) < 1 / (1 + np.exp(-eta))).astype(float)
        s = np.bincount(ind, weights=y, minlength=n_ind)
        keep = ((s > 0) & (s < years))[ind]
    _, ind2 = np.unique(ind[keep], return_inverse=True)
    return [(ind2.astype(np.uint32), int(ind2.max()) + 1), (year[keep], years)], y[keep], X[keep]


@pytest.mark.parametrize("family", ["poisson", "logit"])
def test_absorbed_irls_matches_dense(family):
    terms, y, X = panel(3, 150, 6, family)
    vce = "robust"
    b, V, dev, ll, _ = oglm.irls_absorbed([c for c, _ in terms], [g for _, g in terms], y, X, family, vce, tol=1e-12)
    bd, Vd, devd, lld = oglm.dense_glm(family, terms, y, X, vce)
    assert np.max(np.abs(b - bd) / np.maximum(1, np.abs(bd))) <= 1e-7
    assert np.max(np.abs(V - Vd)) <= 1e-6 * np.max(np.abs(Vd))
    assert abs(ll - lld) <= 1e-9 * abs(lld)


def test_absorbed_irls_matches_stata_logit():
    data = load_csv("glm_logit.csv")
    fix = [f for f in load_json("logit_fixtures.json") if f["spec"]["name"] == "l_cluster"][0]
    terms = [oracle.factorize(data[f]) for f in ("fe1", "fe2")]
    cl = oracle.factorize(data["c"])
    X = np.column_stack([data["x1"], data["x2"]])
    b, V, dev, ll, _ = oglm.irls_absorbed([c for c, _ in terms], [g for _, g in terms], data["y"], X, "logit",
                                          "cluster", cl, tol=1e-12)
    assert np.max(np.abs(b - fix["b"]) / np.abs(fix["b"])) <= 1e-7
    Vw = np.array(fix["V"]).reshape(2, 2)
    assert np.max(np.abs(V - Vw)) <= 1e-6 * np.max(np.abs(Vw))
    assert abs(ll - fix["scalars"]["ll"]) <= 1e-7 * abs(fix["scalars"]["ll"])
