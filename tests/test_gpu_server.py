"""The serving engine on the GPU: a mixed stream of OLS, IV and logit requests gives the same
bits as each request run alone on its own session, whatever the concurrency.

Every kernel reduces in a fixed order and a request's work stays on its own stream, so the
results are compared for exact equality: in the mix (4 workers), alone through the server
(1 worker), and through direct session calls with the host-permuted row block.
"""

import numpy as np
import pytest

import fereg_b200 as fb

pytestmark = pytest.mark.gpu


def make_request(seed):
    rng = np.random.default_rng(seed)
    model = ["ols", "ols", "ols", "iv", "logit"][seed % 5]
    n_ind = int(rng.integers(200, 3000))
    years = 10
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    n_firm = max(10, n_ind // 5)
    firm = ((np.arange(n) // 3) % n_firm).astype(np.uint32) if seed % 2 else rng.integers(0, n_firm, n).astype(np.uint32)
    _, firm = np.unique(firm, return_inverse=True)
    firm = firm.astype(np.uint32)
    nfe = 2 + seed % 2
    codes = [ind, year, firm][:nfe]
    g = [n_ind, years, int(firm.max()) + 1][:nfe]
    nx = int(rng.integers(1, 6))
    X = rng.standard_normal((n, nx))
    a = rng.standard_normal(n_ind)[ind]
    cl = (ind // 7).astype(np.uint32)
    if model == "iv":
        Z = rng.standard_normal((n, 2))
        u = rng.standard_normal(n)
        en = Z @ [0.7, -0.4] + 0.5 * u + rng.standard_normal(n) + a
        y = 0.5 * en + X @ np.linspace(0.1, 0.5, nx) + a + u
        cols = [y] + list(X.T) + [en] + list(Z.T)
        kw = dict(nendog=1, ninst=2, vce="robust")
    elif model == "logit":
        eta = X @ np.linspace(0.2, -0.3, nx) + 0.5 * a
        y = (rng.random(n) < 1 / (1 + np.exp(-eta))).astype(float)
        y[0::years] = 1.0  # every individual has both outcomes: no `fe` separation
        y[1::years] = 0.0
        cols = [y] + list(X.T)
        kw = dict(vce="oim")
    else:
        y = X @ np.linspace(1.0, 0.2, nx) + a + rng.standard_normal(n)
        cols = [y] + list(X.T)
        kw = dict(vce=["unadjusted", "robust", "cluster"][seed % 3])
    clusters = [cl] if kw["vce"] == "cluster" else []
    cl_g = [int(cl.max()) + 1] if clusters else []
    return dict(model=model, codes=codes, g=g, cols=cols, nx=nx, clusters=clusters, cl_g=cl_g, kw=kw)


def alone(r):
    sess = fb.Session(r["codes"], r["g"], r["clusters"], r["cl_g"])
    rows = np.ascontiguousarray(np.column_stack(r["cols"])[sess.row_order()])
    if r["model"] == "ols":
        out = sess.ols(rows, vce=r["kw"]["vce"], tol=1e-10)
    elif r["model"] == "iv":
        out = sess.iv(rows, r["nx"], 1, 2, vce=r["kw"]["vce"], tol=1e-10)
    else:
        out = sess.logit(rows, vce="oim", tol=1e-8, inner_maxiter=16000)
    return out["b"], out["V"]


def serve(reqs, workers):
    srv = fb.Server(workers=workers)
    tickets = [srv.submit(r["model"], r["codes"], r["g"], r["cols"], r["nx"], clusters=r["clusters"], cl_g=r["cl_g"],
                          tol=1e-10 if r["model"] != "logit" else 1e-8, **r["kw"]) for r in reqs]
    out = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    return out, st


def test_mixed_stream_matches_requests_alone():
    reqs = [make_request(s) for s in range(15)]
    mixed, st = serve(reqs, 4)
    assert st["completed"] == len(reqs) and st["peak_bytes"] <= st["budget"]
    single, _ = serve(reqs, 1)
    for r, m, s in zip(reqs, mixed, single):
        assert m["rc"] == 0 and s["rc"] == 0, (m["msg"], s["msg"])
        b, V = alone(r)
        assert np.array_equal(m["b"], s["b"]) and np.array_equal(m["V"], s["V"]), r["model"]
        assert np.array_equal(m["b"], b) and np.array_equal(m["V"], V), r["model"]
        assert m["N"] == len(r["cols"][0])
