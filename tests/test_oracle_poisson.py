"""The oracle's absorbed Poisson IRLS (oracle/glm.py) against the reference's frozen ppmlhdfe
2.3.3 fixtures (tests/golden/poisson_fixtures.json; the reference's harness tests/glm.rs:432-480).

Tolerances are the harness's: b 1e-7 and V 1e-6 relative on the regressors' block (the fixtures'
_cons is a normalization of the absorbed FE, which this path does not report), ll and deviance
1e-6, the sample, N, N_clust and the singleton count exact, and the omitted regressors (o.
columns) omitted here too. The two-way cluster fixture compares everything but V (its spec says
why).
"""

import numpy as np
import pytest

from oracle import glm as oglm
from tests._fixtures import load_poisson, prepare_poisson

FIXTURES, DATA = load_poisson()


def close(a, b, tol):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return np.all(np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-300) + 1e-300)


def expected(fx):
    k = len(fx["spec"]["x"])
    p = len(fx["b"])
    b = np.array(fx["b"][:k], dtype=float)
    V = np.array(fx["V"], dtype=float).reshape(p, p)[:k, :k]
    omitted = [c.startswith("o.") for c in fx["colnames"].split()[:k]]
    return b, V, np.array(omitted)


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_matches_ppmlhdfe(fx):
    spec = fx["spec"]
    keep, nsing, terms, cl, block = prepare_poisson(spec, DATA[spec["data"]])
    assert np.array_equal(keep, np.array(fx["sample"], dtype=float) == 1.0)
    sc = fx["scalars"]
    assert block.shape[0] == sc["N"] and nsing == sc["num_singletons"] and sc["num_separated"] == 0
    codes, g = [c for c, _ in terms], [n for _, n in terms]
    b, V, dev, ll, _ = oglm.irls_absorbed(codes, g, block[:, 0], block[:, 1:], "poisson", spec["vce"],
                                          cl if cl else None, tol=spec["tol"], itol=1e-9)
    bw, Vw, omitted = expected(fx)
    se = np.sqrt(np.maximum(np.diag(V), 0))
    assert np.array_equal(se == 0, omitted)
    kept = ~omitted
    assert close(b[kept], bw[kept], 1e-7), (b, bw)
    if spec.get("compare_v", True):
        assert close(V[np.ix_(kept, kept)], Vw[np.ix_(kept, kept)], 1e-6), (V, Vw)
    assert close(ll, sc["ll"], 1e-6) and close(dev, sc["deviance"], 1e-6)
    if sc.get("N_clust") is not None:
        assert min(G for _, G in cl) == sc["N_clust"]
