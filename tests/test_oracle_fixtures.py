"""Pins the CPU oracle against the reference's frozen reghdfe 6.13.1 fixtures.

Tolerances and checks follow the reference's harness (crates/fereg-core/tests/ols.rs:912-953):
b rtol 1e-7, V rtol 1e-6, dof_table / sample / integer scalars exact, float scalars 1e-6,
resid and d 1e-6, groupvar exact.
"""

import numpy as np
import pytest

from oracle import oracle
from tests._fixtures import load_data, load_fixtures, model_args, nums

DATA = load_data()
FIXTURES = load_fixtures()

INT_SCALARS = ["N", "rank", "df_r", "df_m", "df_a", "df_a_initial", "df_a_redundant", "df_a_nested", "N_clust",
               "N_clustervars", "N_clust1", "N_clust2", "num_singletons", "N_full", "report_constant"]
FLOAT_SCALARS = ["tss", "tss_within", "rss", "mss", "rmse", "F", "ll", "ll_0", "r2", "r2_within", "r2_a",
                 "r2_a_within", "sumweights"]


def close(got, want, rtol):
    got, want = np.asarray(got, float), np.asarray(want, float)
    both_nan = np.isnan(got) & np.isnan(want)
    return bool(np.all(both_nan | (np.abs(got - want) <= rtol * np.maximum(1.0, np.abs(want)))))


@pytest.mark.parametrize("fix", FIXTURES, ids=[f["spec"]["name"] for f in FIXTURES])
def test_oracle_matches_reghdfe(fix):
    spec = fix["spec"]
    args = model_args(spec, DATA)
    res = oracle.ols(**args, tol=1e-14, maxiter=100000, want_resid="r" in fix, want_d="d" in fix,
                     want_groupvar="gv" in fix)
    sample = np.array(fix["sample"], dtype=float)
    assert np.array_equal(res["sample"].astype(float), sample)
    colnames = fix["colnames"].split()
    b, V = res["b"], res["V"]
    k = len(b)
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
    keep = sample == 1.0
    if "r" in fix:
        assert close(res["resid"], nums(fix["r"])[keep], 1e-6)
    if "d" in fix:
        assert close(res["d"], nums(fix["d"])[keep], 1e-6)
    if "gv" in fix:
        assert np.array_equal(res["groupvar"], nums(fix["gv"])[keep])
