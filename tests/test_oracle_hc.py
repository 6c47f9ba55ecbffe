"""The dense HC2 / HC3 oracle (oracle/hc.py) against the reference's frozen Stata 19 `regress ...,
vce(hc2|hc3)` fixtures on vce_cs.csv (harness crates/fereg-core/tests/vce.rs:509-550: b and V of
the x block with i.f1 i.f2, all of them without; tolerance 1e-8, V relative to
sqrt(V_aa V_bb)).
"""

import numpy as np
import pytest

from oracle import hc as ohc
from oracle import oracle
from tests._fixtures import load_csv, load_json
from tests.test_oracle_crv3 import cov_err

DATA = load_csv("vce_cs.csv")
FIXTURES = load_json("hc_fixtures.json")


def prepare_hc(spec):
    terms = [oracle.factorize(DATA[f]) for f in ("f1", "f2")] if spec["absorb"] else []
    w = DATA[spec["weight"]] if spec["weight"] else None
    X = np.column_stack([DATA["x1"], DATA["x2"]])
    return terms, DATA["y"], X, w


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_hc_matches_regress(fx):
    spec = fx["spec"]
    terms, y, X, w = prepare_hc(spec)
    b, V, _ = ohc.hc_ols([c for c, _ in terms], [g for _, g in terms], y, X, spec["hc"] == "hc3", w,
                         spec["weight_kind"])
    p = len(fx["b"])
    bw = np.array(fx["b"], dtype=float)
    Vw = np.array(fx["V"], dtype=float).reshape(p, p)
    assert np.max(np.abs(b[:p] - bw) / np.abs(bw)) <= 1e-8, (b, bw)
    assert cov_err(V[:p, :p], Vw) <= 1e-8, (V[:p, :p], Vw)
