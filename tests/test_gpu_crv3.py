"""CRV3 of the device OLS (fereg_session_ols, vce 3: crv3.rs on the device session) against the
reference's frozen CRV3 fixtures (vce_crv3_ols_{nested,aw,c2,twoway}.json on vce_cs.csv; harness
crates/fereg-core/tests/vce.rs:557-615): b and V of [x1, x2, _cons] at 1e-8 (V relative to
sqrt(V_aa V_bb)), N_clust and df_r exact. The nested fixtures take the closed form (every FE term
nested in the cluster), the others the refits; both paths also agree with the dense oracle.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import crv3 as ocrv3
from oracle import slopes as osl
from tests.test_oracle_crv3 import FIXTURES, cov_err, prepare_crv3

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fx", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_crv3_matches_fixture(fx):
    spec = fx["spec"]
    alive, terms, clusters, y, X, w = prepare_crv3(spec)
    codes, g = [c for c, _ in terms], [n for _, n in terms]
    sess = fb.Session(codes, g, [c for c, _ in clusters], [n for _, n in clusters], w, spec["weight_kind"])
    pi = sess.row_order()
    rows = np.ascontiguousarray(np.column_stack([y, X])[pi])
    res = sess.ols(rows, vce="crv3", tol=1e-14, maxiter=100000)
    sess.close()
    bw = np.array(fx["b"], dtype=float)
    Vw = np.array(fx["V"], dtype=float).reshape(len(bw), len(bw))
    assert np.max(np.abs(res["b"] - bw) / np.abs(bw)) <= 1e-8, (res["b"], bw)
    assert cov_err(res["V"], Vw) <= 1e-8, (res["V"], Vw)
    assert res["scalars"]["N_clust"] == fx["scalars"]["N_clust"]
    assert res["scalars"]["df_r"] == fx["scalars"]["df_r"]
    slots, df_a = osl.estimate_dof(codes, g, [True] * len(codes), [[] for _ in codes], [c for c, _ in clusters])
    _, Vo = ocrv3.crv3_ols(codes, g, y, X, clusters, df_a, any(s[3] for s in slots), w)
    assert cov_err(res["V"], Vo) <= 1e-9
