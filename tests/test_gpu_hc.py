"""HC2 / HC3 of the device OLS (fereg_session_ols, vce 4 / 5: the exact FE leverage of
leverage.rs:128 on the device, ols.rs:450-474) against the reference's frozen Stata 19 `regress
..., vce(hc2|hc3)` fixtures on vce_cs.csv (harness crates/fereg-core/tests/vce.rs:509-550): b and V
of the x block at 1e-8 (V relative to sqrt(V_aa V_bb)), all of b and V without absorbed terms, N
and df_r exact; and the same against the dense oracle (oracle/hc.py).
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import hc as ohc
from tests.test_oracle_crv3 import cov_err
from tests.test_oracle_hc import FIXTURES, prepare_hc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_hc_matches_regress(fx):
    spec = fx["spec"]
    terms, y, X, w = prepare_hc(spec)
    n = len(y)
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms], (), (), w, spec["weight_kind"], n=n)
    pi = sess.row_order()
    rows = np.ascontiguousarray(np.column_stack([y, X])[pi])
    res = sess.ols(rows, vce=spec["hc"], tol=1e-14, maxiter=100000)
    sess.close()
    p = len(fx["b"])
    bw = np.array(fx["b"], dtype=float)
    Vw = np.array(fx["V"], dtype=float).reshape(p, p)
    assert np.max(np.abs(res["b"][:p] - bw) / np.abs(bw)) <= 1e-8, (res["b"], bw)
    assert cov_err(res["V"][:p, :p], Vw) <= 1e-8, (res["V"], Vw)
    assert res["scalars"]["N"] == fx["scalars"]["N"]
    assert res["scalars"]["df_r"] == fx["scalars"]["df_r"]
    _, Vo, _ = ohc.hc_ols([c for c, _ in terms], [g for _, g in terms], y, X, spec["hc"] == "hc3", w,
                          spec["weight_kind"])
    assert cov_err(res["V"][:p, :p], Vo[:p, :p]) <= 1e-9
