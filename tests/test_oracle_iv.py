"""The oracle's 2SLS restatement (oracle/iv.py) against the reference's ivreghdfe fixtures.

Pins the oracle before it checks the device IV: 32 fixtures (nlswork subset,
`ln_wage age (tenure = union south [msp])`, absorb(idcode year), unadjusted / robust / cluster
idcode / cluster idcode year x none / aw / fw / pw; tests/iv.rs:216-248 of the reference).
Tolerances of the reference's harness (tests/iv.rs:365-370): b 1e-7, V 1e-6 relative.
"""

import numpy as np
import pytest

from oracle import iv as oiv
from tests._fixtures import iv_block, load_csv, load_json, prepare_iv

DATA = load_csv("iv_nls.csv")
FIXTURES = load_json("iv_fixtures.json")


@pytest.mark.parametrize("fix", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_iv_matches_ivreghdfe(fix):
    spec = fix["spec"]
    alive, nsing, terms, clusters, w = prepare_iv(spec, DATA)
    assert np.array_equal(alive.astype(float), np.array(fix["sample"], dtype=float))
    Y = iv_block(spec, DATA, alive)
    Yt = oiv.residualize([c for c, _ in terms], [g for _, g in terms], Y, w)
    b, V, rss, big_n = oiv.tsls(Yt, len(spec["exog"]), len(spec["endog"]), len(spec["inst"]), w, spec["weight_kind"],
                                spec["vce"], [c for c, _ in clusters], fix["scalars"]["df_a"])
    bw = np.array(fix["b"])
    Vw = np.array(fix["V"]).reshape(V.shape)
    assert np.max(np.abs(b - bw) / np.abs(bw)) <= 1e-7
    assert np.max(np.abs(V - Vw)) <= 1e-6 * np.max(np.abs(Vw))
    assert abs(rss - fix["scalars"]["rss"]) <= 1e-9 * rss
    assert big_n == fix["scalars"]["N"]
