"""The oracle's dense logit (oracle/glm.py) against the reference's Stata logit fixtures.

Stata `logit y x1 x2 i.fe1 i.fe2` (and `i.fe1` alone) at tol(1e-12) ltol(1e-14) on
glm_logit.csv (the reference's tests/glm.rs:659-672): the slopes' b and V (oim, robust, cluster
c) and the log-likelihood. Tolerances of the reference's harness (tests/glm.rs:535-545): b 1e-7,
V 1e-6, ll 1e-7 relative.
"""

import numpy as np
import pytest

from oracle import glm as oglm
from oracle import oracle
from tests._fixtures import load_csv, load_json

DATA = load_csv("glm_logit.csv")
FIXTURES = load_json("logit_fixtures.json")


def logit_case(spec):
    terms = [oracle.factorize(DATA[f]) for f in spec["absorb"]]
    cl = oracle.factorize(DATA[spec["cluster"]]) if spec["cluster"] else None
    X = np.column_stack([DATA["x1"], DATA["x2"]])
    return terms, DATA["y"], X, cl


@pytest.mark.parametrize("fix", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_logit_matches_stata(fix):
    spec = fix["spec"]
    assert all(s == 1 for s in fix["sample"])
    terms, y, X, cl = logit_case(spec)
    b, V, dev, ll = oglm.dense_glm("logit", terms, y, X, spec["vce"], cl)
    bw = np.array(fix["b"])
    Vw = np.array(fix["V"]).reshape(2, 2)
    assert np.max(np.abs(b - bw) / np.abs(bw)) <= 1e-7
    assert np.max(np.abs(V - Vw)) <= 1e-6 * np.max(np.abs(Vw))
    assert abs(ll - fix["scalars"]["ll"]) <= 1e-7 * abs(fix["scalars"]["ll"])
    assert abs(dev + 2 * fix["scalars"]["ll"]) <= 1e-7 * abs(dev)
