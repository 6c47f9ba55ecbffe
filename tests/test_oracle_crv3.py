"""The dense CRV3 oracle (oracle/crv3.py) against the reference's frozen CRV3 fixtures for OLS
(do-file jackknife loops of reghdfe over vce_cs.csv: vce_crv3_ols_{nested,aw,c2,twoway}.json;
harness crates/fereg-core/tests/vce.rs:557-615, tolerance 1e-8 on b and on V relative to
sqrt(V_aa V_bb), ols/stata_vce.rs:516-545 for the multiway meat). The dof (df_a, nested) comes
from the slope oracle's estimate_dof with the clusters, as reghdfe computes it.
"""

import numpy as np
import pytest

from oracle import crv3 as ocrv3
from oracle import oracle
from oracle import slopes as osl
from tests._fixtures import load_csv, load_json

DATA = load_csv("vce_cs.csv")
FIXTURES = load_json("crv3_fixtures.json")


def cov_err(got, want):
    """tests/vce.rs:259-270."""
    p = want.shape[0]
    e = 0.0
    for a in range(p):
        for b in range(p):
            s = np.sqrt(abs(want[a, a] * want[b, b]))
            d = abs(got[a, b] - want[a, b])
            e = max(e, 0.0 if d == 0 else d / max(s, abs(want[a, b])))
    return e


def prepare_crv3(spec):
    fac = {f: oracle.factorize(DATA[f]) for f in set(spec["absorb"]) | set(spec["cluster"])}
    terms = [fac[f] for f in spec["absorb"]]
    w = DATA[spec["weight"]] if spec["weight"] else None
    alive, nsing = oracle.drop_singletons([c for c, _ in terms], [g for _, g in terms],
                                          w if spec["weight_kind"] == "fweight" else None)

    def restrict(c):
        u, inv = np.unique(c[alive], return_inverse=True)
        return inv.astype(np.uint32), len(u)

    terms = [restrict(c) for c, _ in terms]
    clusters = [restrict(fac[f][0]) for f in spec["cluster"]]
    X = np.column_stack([DATA[x][alive] for x in spec["x"]])
    return alive, terms, clusters, DATA[spec["y"]][alive], X, (None if w is None else w[alive])


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_crv3_matches_fixture(fx):
    spec = fx["spec"]
    alive, terms, clusters, y, X, w = prepare_crv3(spec)
    assert int(alive.sum()) == fx["scalars"]["N"]
    codes, g = [c for c, _ in terms], [n for _, n in terms]
    slots, df_a = osl.estimate_dof(codes, g, [True] * len(codes), [[] for _ in codes], [c for c, _ in clusters])
    assert df_a == fx["scalars"]["df_a"]
    nested = any(s[3] for s in slots)
    theta, V = ocrv3.crv3_ols(codes, g, y, X, clusters, df_a, nested, w)
    bw = np.array(fx["b"], dtype=float)
    assert np.max(np.abs(theta - bw) / np.abs(bw)) <= 1e-8
    Vw = np.array(fx["V"], dtype=float).reshape(len(bw), len(bw))
    assert cov_err(V, Vw) <= 1e-8, (V, Vw)
