"""The oracle's ReLU separation check (oracle/glm.py relu_separation) in the reference's rounds
(tests/_fixtures.py prepare_separation) against the ppmlhdfe 2.3.3 fixtures fitted with
sep(fe relu) (tests/golden/separation_fixtures.json; harness crates/fereg-core/tests/glm.rs:
432-480, 549-590): the sample exactly, N, the separated and singleton counts (the harness's
where it overrides them), and, where the fixture has regressors, the Poisson b on them at 1e-7
under the harness's rule (tests/glm.rs:171-185; the oracle's absorbed IRLS on the prepared
sample) with the omitted ones omitted.
"""

import numpy as np
import pytest

from oracle import glm as oglm
from tests._fixtures import load_separation, prepare_separation


def close_h(got, want, rtol):
    """The harness's vector rule (tests/glm.rs:171-185): |a - b| <= rtol (atol / rtol +
    max(|a|, |b|)) with atol = 1e-10 max |want| + 1e-14."""
    got, want = np.asarray(got, dtype=float), np.asarray(want, dtype=float)
    atol = 1e-10 * np.abs(want[np.isfinite(want)]).max(initial=0.0) + 1e-14
    return bool(np.all(np.abs(got - want) <= rtol * (atol / rtol + np.maximum(np.abs(got), np.abs(want)))))

FIXTURES, DATA = load_separation()


def oracle_check(terms, block):
    sep, complete = oglm.relu_separation([c for c, _ in terms], [g for _, g in terms], block[:, 0], block[:, 1:])
    assert complete
    return sep


def expected_counts(fx):
    sc = fx["scalars"]
    return tuple(fx["spec"]["counts"]) if fx["spec"]["counts"] else (sc["num_separated"], sc["num_singletons"])


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_separation_matches_ppmlhdfe(fx):
    spec = fx["spec"]
    keep, nsep, nsing, terms, block = prepare_separation(spec, DATA[spec["data"]], oracle_check)
    assert np.array_equal(keep, np.array(fx["sample"], dtype=float) == 1.0)
    assert block.shape[0] == fx["scalars"]["N"]
    assert (nsep, nsing) == expected_counts(fx)
    k = len(spec["x"])
    if k:
        b, V, dev, ll, _ = oglm.irls_absorbed([c for c, _ in terms], [g for _, g in terms], block[:, 0],
                                              block[:, 1:], "poisson", tol=spec["tol"], maxiter=spec["maxiter"])
        omitted = np.array([c.startswith("o.") for c in fx["colnames"].split()[:k]])
        bw = np.array(fx["b"][:k], dtype=float)
        assert np.all(b[omitted] == 0.0)
        assert close_h(b[~omitted], bw[~omitted], 1e-7), (b, bw)
