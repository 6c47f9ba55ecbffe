"""The device OLS (fereg_session_ols) against the reference's frozen reghdfe 6.13.1 fixtures.

The sample preparation (factorize, interactions, drop_singletons, restrict) is done here with the
oracle's preparation functions, as the reference's Session::prepare would; everything after it
(degrees of freedom, column statistics, the FE solve, the Gram, collinearity, coefficients and
variance) runs through the C ABI of the B200 session. Tolerances follow the reference's harness
(crates/fereg-core/tests/ols.rs:912-953): b 1e-7, V 1e-6, dof table and integer scalars exact,
float scalars 1e-6, resid and d 1e-6, groupvar exact.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import oracle
from tests._fixtures import FACTORS, load_data, load_fixtures, nums
from tests.test_oracle_fixtures import FLOAT_SCALARS, INT_SCALARS, close

pytestmark = pytest.mark.gpu

DATA = load_data()
FIXTURES = load_fixtures()


def interact(parts):
    """Codes of the interaction of factor codes (mixed radix, ascending), with its level count."""
    if len(parts) == 1:
        return parts[0]
    key = np.zeros(len(parts[0][0]), dtype=np.uint64)
    for codes, g in parts:
        key = key * np.uint64(g) + codes.astype(np.uint64)
    u, inv = np.unique(key, return_inverse=True)
    return inv.astype(np.uint32), len(u)


def prepare(spec):
    fac = {f: oracle.factorize(DATA[f]) for f in FACTORS}
    terms = [interact([fac[f] for f in t]) for t in spec["absorb"]]
    clusters = [fac[c] for c in spec["vce"]]
    w = DATA[spec["weight"]] if spec["weight"] else None
    fw = w if spec["weight_kind"] == "fweight" else None
    n0 = len(DATA["y"])
    if spec["singletons"] and terms:
        alive, nsing = oracle.drop_singletons([c for c, _ in terms], [g for _, g in terms], fw)
    else:
        alive, nsing = np.ones(n0, dtype=bool), 0

    def restrict(c):
        u, inv = np.unique(c[alive], return_inverse=True)
        return inv.astype(np.uint32), len(u)

    terms = [restrict(c) for c, _ in terms]
    clusters = [restrict(c) for c, _ in clusters]
    return alive, nsing, terms, clusters, (None if w is None else w[alive])


@pytest.mark.parametrize("fix", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_device_ols_matches_reghdfe(fix):
    spec = fix["spec"]
    alive, nsing, terms, clusters, w = prepare(spec)
    sess = fb.Session([c for c, _ in terms], [g for _, g in terms], [c for c, _ in clusters],
                      [g for _, g in clusters], w, spec["weight_kind"], nsing)
    pi = sess.row_order()
    cols = [DATA[spec["y"]][alive]] + [DATA[x][alive] for x in spec["x"]]
    rows = np.ascontiguousarray(np.stack(cols, axis=1)[pi])
    vce = "cluster" if spec["vce"] else ("robust" if spec["robust"] else "unadjusted")
    res = sess.ols(rows, vce=vce, noconstant=spec["noconstant"], firstpair=spec["firstpair"],
                   want_groupvar="gv" in fix, want_resid="r" in fix, want_d="d" in fix, tol=1e-14, maxiter=100000)
    assert np.array_equal(alive.astype(float), np.array(fix["sample"], dtype=float))
    colnames = fix["colnames"].split()
    b, V = res["b"], res["V"]
    for j, name in enumerate(colnames):
        zero = b[j] == 0.0 and V[j, j] == 0.0
        st = res["status"][j] if j < len(res["status"]) else 0
        assert (st != 0 or zero) == name.startswith("o."), name
    if "status" in spec:
        assert list(res["status"]) == spec["status"]
    assert close(b, nums(fix["b"]), 1e-7), (b, fix["b"])
    assert close(V.ravel(), nums(fix["V"]), 1e-6), (V.ravel(), fix["V"])
    assert np.array_equal(res["dof_table"].ravel(), nums(fix["dof_table"]))
    for name, want in fix["scalars"].items():
        if name in ("N_hdfe", "N_hdfe_extended", "drop_singletons", "ic", "converged"):
            continue
        got = res["scalars"][name]
        want = np.nan if want is None else float(want)
        if name in INT_SCALARS:
            assert got == want or (np.isnan(got) and np.isnan(want)), (name, got, want)
        else:
            assert name in FLOAT_SCALARS
            assert close(got, want, 1e-6), (name, got, want)
    keep = alive
    if "r" in fix:
        assert close(res["resid"], nums(fix["r"])[keep], 1e-6)
    if "d" in fix:
        assert close(res["d"], nums(fix["d"])[keep], 1e-6)
    if "gv" in fix:
        assert np.array_equal(res["groupvar"], nums(fix["gv"])[keep])
    assert sess.launches() > 0
