"""The serving engine's scheduler on the host (dry-run server: no GPU).

Requests are admitted in arrival order while their estimated device memory fits the budget, at
most `workers` run at once, a request larger than the whole budget is rejected with the
reference's OutOfMemory code (909), and malformed requests fail with 198.
"""

import time

import numpy as np
import pytest

import fereg_b200 as fb

CODES = [np.zeros(4, dtype=np.uint32)]
COLS = [np.zeros(4)] * 3


def submit(srv, n, us, model="ols", nx=2, **kw):
    return srv.submit(model, CODES, [1], COLS[: 1 + nx + kw.get("nendog", 0) + kw.get("ninst", 0)], nx, n=n,
                      dry_run_us=us, **kw)


def test_fifo_admission_within_budget():
    # the estimate of one request sets the budget: two fit at once, a third does not
    probe = fb.Server(workers=1, hbm_budget=1 << 40, dry_run=True)
    one = probe.wait(submit(probe, 1_000_000, 0))["bytes"]
    probe.close()
    srv = fb.Server(workers=4, hbm_budget=2 * one + one // 2, dry_run=True)
    tickets = [submit(srv, 1_000_000, 20_000) for _ in range(10)]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert st["completed"] == 10 and st["rejected"] == 0
    assert st["peak_bytes"] <= st["budget"] and st["peak_running"] == 2
    admits = [r["admit_s"] for r in res]
    assert admits == sorted(admits)  # first in, first admitted
    assert all(r["rc"] == 0 and r["done_s"] >= r["admit_s"] >= r["submit_s"] for r in res)


def test_workers_bound_concurrency():
    srv = fb.Server(workers=3, hbm_budget=1 << 50, dry_run=True)
    t0 = time.perf_counter()
    res = [srv.wait(t) for t in [submit(srv, 1000, 50_000) for _ in range(9)]]
    wall = time.perf_counter() - t0
    st = srv.stats()
    assert st["peak_running"] == 3 and st["completed"] == 9
    assert 0.14 <= wall < 1.0, wall  # three waves of 50 ms
    assert max(r["done_s"] for r in res) - min(r["admit_s"] for r in res) >= 0.14


def test_head_of_line_blocks_smaller_requests():
    """A large request at the head waits for memory; smaller ones behind it do not overtake."""
    probe = fb.Server(workers=1, hbm_budget=1 << 40, dry_run=True)
    big = probe.wait(submit(probe, 4_000_000, 0))["bytes"]
    probe.close()
    srv = fb.Server(workers=4, hbm_budget=big + big // 4, dry_run=True)
    a = submit(srv, 1_000_000, 60_000)
    b = submit(srv, 4_000_000, 10_000)
    c = submit(srv, 10_000, 0)
    ra, rb, rc = srv.wait(a), srv.wait(b), srv.wait(c)
    assert rb["admit_s"] >= ra["done_s"] - 1e-3  # b needed a's memory
    assert rc["admit_s"] >= rb["admit_s"]


def test_request_larger_than_budget_is_rejected():
    srv = fb.Server(workers=2, hbm_budget=64 << 20, dry_run=True)
    with pytest.raises(fb.FeregError) as e:
        submit(srv, 50_000_000, 0)
    assert e.value.rc == 909
    assert srv.stats()["rejected"] == 1
    assert srv.wait(submit(srv, 1000, 0))["rc"] == 0


def test_malformed_requests_are_refused():
    srv = fb.Server(workers=1, hbm_budget=1 << 40, dry_run=True)
    with pytest.raises(fb.FeregError) as e:
        srv.submit("iv", CODES, [1], COLS[:3], 2, n=4)  # IV without an endogenous regressor
    assert e.value.rc == 198
    with pytest.raises(fb.FeregError) as e:
        srv.submit("ols", CODES, [1], COLS[:3], 1, nendog=1, n=4)  # endogenous columns outside IV
    assert e.value.rc == 198
    with pytest.raises(fb.FeregError):
        srv.wait(12345)


def test_dry_run_needs_a_budget():
    with pytest.raises(fb.FeregError) as e:
        fb.Server(workers=1, hbm_budget=None, dry_run=True)
    assert e.value.rc == 198


def test_estimate_counts_the_dense_small_block():
    """A request whose small super-block gets the dense factor (900 coordinates <= 1024) is
    estimated ~62 MB above one whose small block is too large for it (1100 coordinates): the
    factor, its work arrays and inverse (4 ms^2 doubles) and the assembly rows ((4096 + ms) ms)."""
    srv = fb.Server(workers=1, hbm_budget=1 << 40, dry_run=True)
    est = {}
    for levels in (900, 1100):
        t = srv.submit("ols", CODES * 2, [5000, levels], COLS, 2, n=100_000, dry_run_us=0)
        est[levels] = srv.wait(t)["bytes"]
    srv.close()
    dense = (4 * 900 * 900 + (4096 + 900) * 900) * 8
    assert est[900] - est[1100] == dense - 200 * 3 * 8 * 10
