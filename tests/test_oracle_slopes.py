"""The dense slope oracle (oracle/slopes.py) pinned to the reference's reghdfe fixture with a
slope term: ols_s16_slopes (reghdfe y x1 x2, absorb(id firm##c.x4); harness
crates/fereg-core/tests/ols.rs:827, tolerances of tests/ols.rs:912-953: b 1e-7, V 1e-6, dof table
and integer scalars exact). Plus the oracle's own invariants on a random panel: the residuals are
orthogonal to every design column, and projecting twice changes nothing.
"""

import json
import os

import numpy as np

from oracle import oracle
from oracle import slopes as osl
from tests._fixtures import GOLDEN, load_data, nums
from tests.test_oracle_fixtures import close


def load_slope_fixtures():
    with open(os.path.join(GOLDEN, "ols_slopes_fixtures.json")) as f:
        return json.load(f)


def prepare_slopes(spec, data):
    """Factorize, drop singletons on the terms' factors, restrict; the slope variables follow."""
    fac = {f: oracle.factorize(data[f]) for t in spec["absorb"] for f in t}
    terms = [fac[t[0]] for t in spec["absorb"]]
    alive, nsing = oracle.drop_singletons([c for c, _ in terms], [g for _, g in terms])

    def restrict(c):
        u, inv = np.unique(c[alive], return_inverse=True)
        return inv.astype(np.uint32), len(u)

    terms = [restrict(c) for c, _ in terms]
    slopes = [[data[x][alive] for x in sl] for sl in spec["term_slopes"]]
    return alive, nsing, terms, slopes


def test_oracle_matches_reghdfe_s16():
    data = load_data()
    fix = load_slope_fixtures()[0]
    spec = fix["spec"]
    alive, nsing, terms, slopes = prepare_slopes(spec, data)
    assert np.array_equal(alive.astype(float), np.array(fix["sample"], dtype=float))
    assert nsing == fix["scalars"]["num_singletons"]
    codes, g = [c for c, _ in terms], [gq for _, gq in terms]
    y = data[spec["y"]][alive]
    X = [data[x][alive] for x in spec["x"]]
    b, V, slots, df_a = osl.ols_iid(codes, g, spec["intercept"], slopes, y, X)
    assert close(b, nums(fix["b"]), 1e-7), (b, fix["b"])
    assert close(V.ravel(), nums(fix["V"]), 1e-6)
    table = np.array([[k, m, k - m, 0 if ex else 1, 1 if ne else 0] for k, m, ex, ne in slots], dtype=float)
    assert np.array_equal(table.ravel(), nums(fix["dof_table"]))
    assert df_a == fix["scalars"]["df_a"]


def test_oracle_projection_invariants():
    rng = np.random.default_rng(5)
    n, ni, nf = 600, 60, 12
    indiv = np.repeat(np.arange(ni), n // ni).astype(np.uint32)
    firm = rng.integers(0, nf, n).astype(np.uint32)
    x = rng.normal(size=n)
    w = 0.5 + rng.random(n)
    codes, g = [indiv, firm], [ni, nf]
    icpt, sl = [True, False], [[], [x]]
    Z = rng.normal(size=(n, 3))
    r = osl.residualize(codes, g, icpt, sl, Z, w)
    D = osl.design(codes, g, icpt, sl)
    assert np.abs(D.T @ (w[:, None] * r)).max() < 1e-9 * np.abs(Z).sum()
    assert np.allclose(osl.residualize(codes, g, icpt, sl, r, w), r, atol=1e-10)
