"""The device ReLU separation check (fereg_session_relu, glm/separation.rs:61-196) in the
reference's rounds against the ppmlhdfe 2.3.3 fixtures fitted with sep(fe relu)
(tests/golden/separation_fixtures.json; harness crates/fereg-core/tests/glm.rs:432-480, 549-590).

Every round prepares the sample on the device (fereg_drop_singletons with the Poisson `fe` rule,
fereg_restrict), builds the session and runs the check through the C ABI; the rows it separates
leave and the next round prepares the rest. Checked: the fixture's e(sample) exactly, N, the
separated and singleton counts (the harness's where it overrides them), the device check's
separated rows equal to the oracle's on the same sample, and where the fixture has regressors the
device Poisson fit's b at 1e-7 under the harness's rule with the omitted regressors omitted.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import glm as oglm
from tests._fixtures import load_separation, prepare_separation
from tests.test_oracle_separation import close_h, expected_counts

pytestmark = pytest.mark.gpu

FIXTURES, DATA = load_separation()


def device_drop(codes, g, y, keepsing):
    alive, _, _ = fb.drop_singletons(codes, g, y=y, family="poisson", singletons=not keepsing)
    return alive


def device_check(terms, block):
    codes, g = [c for c, _ in terms], [n for _, n in terms]
    sess = fb.Session(codes, g)
    pi = sess.row_order()
    out = sess.relu_separation(np.ascontiguousarray(block[pi]))
    sess.close()
    assert out["complete"]
    sep = np.zeros(len(block), dtype=bool)
    sep[pi] = out["separated"]
    # the oracle's check on the same sample finds the same rows
    want, _ = oglm.relu_separation(codes, g, block[:, 0], block[:, 1:])
    assert np.array_equal(sep, want)
    assert out["num_separated"] == int(sep.sum())
    return sep


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_separation_matches_ppmlhdfe(fx):
    spec = fx["spec"]
    keep, nsep, nsing, terms, block = prepare_separation(spec, DATA[spec["data"]], device_check, device_drop)
    assert np.array_equal(keep, np.array(fx["sample"], dtype=float) == 1.0)
    assert block.shape[0] == fx["scalars"]["N"]
    assert (nsep, nsing) == expected_counts(fx)
    k = len(spec["x"])
    if k:
        sess = fb.Session([c for c, _ in terms], [g for _, g in terms])
        rows = np.ascontiguousarray(block[sess.row_order()])
        out = sess.poisson(rows, vce="robust", tol=spec["tol"], maxiter=spec["maxiter"], itol=1e-9)
        sess.close()
        omitted = np.array([c.startswith("o.") for c in fx["colnames"].split()[:k]])
        assert np.array_equal(out["status"] != 0, omitted)
        bw = np.array(fx["b"][:k], dtype=float)
        assert close_h(out["b"][~omitted], bw[~omitted], 1e-7), (out["b"], bw)
