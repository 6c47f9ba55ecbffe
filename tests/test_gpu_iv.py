"""The device IV / 2SLS (fereg_session_iv) against the reference's ivreghdfe fixtures and the oracle.

The sample preparation (factorize, drop_singletons, restrict) uses the oracle's preparation
functions; the one residualization of [y, exog, endog, inst], the degrees of freedom, the Gram,
collinearity, 2SLS and the variance run through the C ABI of the B200 session. Tolerances of the
reference's harness (tests/iv.rs:365-370): b 1e-7, V 1e-6 relative, integer scalars exact.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import iv as oiv
from tests._fixtures import iv_block, load_csv, load_json, prepare_iv

pytestmark = pytest.mark.gpu

DATA = load_csv("iv_nls.csv")
FIXTURES = load_json("iv_fixtures.json")
INT_SCALARS = ("N", "df_r", "df_m", "df_a", "sdofminus", "N_clust", "endog_ct", "inexog_ct", "exexog_ct")


@pytest.mark.parametrize("fix", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_iv_matches_ivreghdfe(fix):
    spec = fix["spec"]
    alive, nsing, terms, clusters, w = prepare_iv(spec, DATA)
    assert np.array_equal(alive.astype(float), np.array(fix["sample"], dtype=float))
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms], [c for c, _ in clusters],
                      [g for _, g in clusters], w, spec["weight_kind"], nsing)
    rows = np.ascontiguousarray(iv_block(spec, DATA, alive)[sess.row_order()])
    res = sess.iv(rows, len(spec["exog"]), len(spec["endog"]), len(spec["inst"]), vce=spec["vce"], tol=1e-14,
                  maxiter=100000)
    assert not res["status"].any()
    bw = np.array(fix["b"])
    Vw = np.array(fix["V"]).reshape(res["V"].shape)
    assert np.max(np.abs(res["b"] - bw) / np.abs(bw)) <= 1e-7, (res["b"], bw)
    assert np.max(np.abs(res["V"] - Vw)) <= 1e-6 * np.max(np.abs(Vw)), (res["V"], Vw)
    for name, want in fix["scalars"].items():
        got = res["scalars"][name]
        if want is None:
            assert np.isnan(got), name
        elif name in INT_SCALARS:
            assert got == want, (name, got, want)
        else:
            assert abs(got - want) <= 1e-6 * abs(want), (name, got, want)


def synthetic(seed, n_ind, years, n_firm, G):
    rng = np.random.default_rng(seed)
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    firm = (np.arange(n) % n_firm).astype(np.uint32)
    cl = rng.integers(0, G, n).astype(np.uint32)
    _, cl = np.unique(cl, return_inverse=True)
    z = rng.standard_normal((n, 2))
    x = rng.standard_normal((n, 2))
    u = rng.standard_normal(n)
    endog = z @ [0.8, -0.5] + 0.3 * x[:, 0] + 0.6 * u + rng.standard_normal(n) + rng.standard_normal(n_ind)[ind]
    y = 0.7 * endog + x @ [0.2, -0.1] + u + rng.standard_normal(n_firm)[firm]
    terms = [(ind, n_ind), (year, years), (firm, n_firm)]
    return terms, np.column_stack([y, x, endog, z]), (cl.astype(np.uint32), int(cl.max()) + 1)


@pytest.mark.parametrize("vce", ["unadjusted", "robust", "cluster"])
def test_device_iv_matches_oracle_three_fe(vce):
    terms, block, (cl, G) = synthetic(11, 400, 8, 97, 60)
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms], [cl], [G])
    rows = np.ascontiguousarray(block[sess.row_order()])
    res = sess.iv(rows, 2, 1, 2, vce=vce, tol=1e-13, maxiter=100000)
    Yt = oiv.residualize([c for c, _ in terms], [g for _, g in terms], block)
    b, V, rss, _ = oiv.tsls(Yt, 2, 1, 2, vce=vce, clusters=[cl], df_a=int(res["scalars"]["df_a"]))
    assert np.max(np.abs(res["b"] - b) / np.maximum(1.0, np.abs(b))) <= 1e-8
    assert np.max(np.abs(res["V"] - V)) <= 1e-7 * np.max(np.abs(V))
    assert abs(res["scalars"]["rss"] - rss) <= 1e-9 * rss


def test_device_iv_not_identified():
    """The only excluded instrument duplicates an exogenous regressor: stage-2 collinearity drops
    it, no excluded instrument is left for the endogenous regressor, and the call fails with the
    reference's code 481 (iv.rs:493-500)."""
    terms, block, (cl, G) = synthetic(12, 100, 5, 13, 10)
    block = np.column_stack([block[:, :4], block[:, 1]])  # [y, x1, x2, endog, z := x1]
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms])
    rows = np.ascontiguousarray(block[sess.row_order()])
    with pytest.raises(fb.FeregError) as e:
        sess.iv(rows, 2, 1, 1)
    assert e.value.rc == 481
