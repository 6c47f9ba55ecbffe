"""The device Poisson PML (fereg_session_poisson) against the reference's frozen ppmlhdfe 2.3.3
fixtures (tests/golden/poisson_fixtures.json; the reference's harness tests/glm.rs:432-480).

The sample preparation runs on the device too (fereg_drop_singletons with the Poisson `fe` rule,
fereg_restrict) and must reproduce the fixture's e(sample) and its drop count; the fit then runs
through the C ABI of the device session. Tolerances are the harness's: b 1e-7 and V 1e-6
relative on the regressors' block, ll and deviance 1e-6, N and N_clust exact, and the omitted
regressors omitted. The two-way cluster fixture compares everything but V (its spec says why).
"""

import numpy as np
import pytest

import fereg_b200 as fb
from tests._fixtures import _interact, load_poisson, prepare_poisson
from tests.test_oracle_poisson import close, expected

pytestmark = pytest.mark.gpu

FIXTURES, DATA = load_poisson()


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_poisson_matches_ppmlhdfe(fx):
    spec = fx["spec"]
    data = DATA[spec["data"]]
    keep, nsing, terms, cl, block = prepare_poisson(spec, data)
    sc = fx["scalars"]
    # the device preparation of the same rows
    base = np.ones(len(data[spec["y"]]), dtype=bool)
    base[[i - 1 for i in spec["exclude"]]] = False
    fac = {f: fb.factorize(data[f][base]) for f in {f for t in spec["absorb"] for f in t}}
    raw_terms = [_interact([fac[f] for f in t]) for t in spec["absorb"]]
    alive, s, f = fb.drop_singletons([c for c, _ in raw_terms], [g for _, g in raw_terms], y=data[spec["y"]][base],
                                     family="poisson", singletons=not spec["keepsing"])
    assert np.array_equal(alive, keep[base]) and s + f == sc["num_singletons"]
    dev_terms = [fb.restrict(c, g, alive) for c, g in raw_terms]
    for (a, ga), (b_, gb) in zip(dev_terms, terms):
        assert ga == gb and np.array_equal(a, b_)

    codes, g = [c for c, _ in terms], [n for _, n in terms]
    sess = fb.Session(codes, g, [c for c, _ in cl], [n for _, n in cl])
    rows = np.ascontiguousarray(block[sess.row_order()])
    out = sess.poisson(rows, vce=spec["vce"], tol=spec["tol"], itol=1e-9)
    sess.close()
    assert out["converged"] and out["N"] == sc["N"]
    bw, Vw, omitted = expected(fx)
    assert np.array_equal(out["status"] != 0, omitted)
    kept = ~omitted
    assert close(out["b"][kept], bw[kept], 1e-7), (out["b"], bw)
    if spec.get("compare_v", True):
        assert close(out["V"][np.ix_(kept, kept)], Vw[np.ix_(kept, kept)], 1e-6), (out["V"], Vw)
    assert close(out["ll"], sc["ll"], 1e-6) and close(out["deviance"], sc["deviance"], 1e-6)
    if sc.get("N_clust") is not None:
        assert out["N_clust"] == sc["N_clust"]
