"""Benchmark of the B200 OLS call on the 1e7-observation 3-FE panel (and the 1e5 2-FE panel).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--config c2|c1]
                    [--precision f64|f32r]

One step is one OLS call (Session::ols, ols.rs:199-470) on a prepared session: degrees of
freedom (mobility groups of the FE pairs), column statistics of the raw block, the FE solve of
[y, x1..x10] against indiv + firm + year, the weighted Gram, collinearity, coefficients, the
residuals and the iid variance. The session (the cell structure, built once from the FE codes)
is prepared outside the timed region; its time is reported as `config.prepare_s`.

`value` times the call with the n x R block already resident in HBM (a fresh copy before each
call, outside the events); `e2e` times the same call through the C ABI with the block in pinned
host memory: the host-to-device copy of the block and the copies of the results to the host are
inside the timed region. Inputs (880 MB) exceed the 126 MB L2, so no flush runs between steps.

Multi-GPU (torchrun): independent replicas, one per GPU (a single solve does not shard at this
size); the step time is the max over ranks and `value` is seconds per call of the whole job.

`--impl reference` times the reference's algorithm on the host cores: the CPU oracle (a C++
restatement of the reference's session OLS; the reference's Rust crate cannot be built here),
with all host threads, on the same prepared session, workload, metric and unit.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # OLS y ~ x1..x10 | indiv + firm + year, n = 1e6 indiv x 10 years, firm = row mod 1e5.
    "c2": dict(n_ind=1_000_000, years=10, n_firm=100_000, k=10, seed=10**7 * 100 + 43),
    # The same OLS on the connected "difficult" firm graph of the reference's benchmark DGP
    # (bench/dgp.py:55,70): n_ind / 23 = 43,478 firms, firm = row mod 43,478. 43,478 is not a
    # multiple of 10, so the individuals' runs of 10 consecutive firms wrap into one ring.
    "c2d": dict(n_ind=1_000_000, years=10, n_firm=43_478, k=10, seed=10**7 * 100 + 47),
    # The C2 shape at 3e6 rows (3e5 indiv x 10 years, firm = row mod 3e4; 264 MB of rows, above
    # L2): the case of the full ncu captures, which must stay a few GB on the device.
    "c2p": dict(n_ind=300_000, years=10, n_firm=30_000, k=10, seed=10**7 * 100 + 45),
    # OLS y ~ x1 | indiv + year, n = 1e4 indiv x 10 years.
    "c1": dict(n_ind=10_000, years=10, n_firm=0, k=1, seed=10**5 * 100 + 42),
    # WCR11 wild cluster bootstrap of b_x1 (H0 true): y ~ x1 | indiv + year + firm, cluster firm,
    # n = 1e5 indiv x 10 years, firm random in 2e4, 9,999 Rademacher draws (seed 1).
    "c3": dict(n_ind=100_000, years=10, n_firm=20_000, k=1, seed=10**6 * 100 + 44, reps=9_999),
    # Poisson PML (gravity): trade ~ x1 + log dist | exporter#year + importer#year + pair, 200
    # countries x 50 years, 39,800 directed pairs x 5 rows (sectors) per pair-year, ~40% zeros,
    # robust SEs.
    "c4": dict(countries=200, years=50, sectors=5, seed=10**7 * 100 + 45, zero_share=0.40),
    # Serving stream: 2,000 requests, exponential inter-arrivals at 70% of the measured capacity,
    # n log-uniform in 1e4..5e6, 1-4 FEs, 60% OLS / 20% IV / 20% logit, 1-12 regressors.
    "c5": dict(requests=2000, seed=10**6 * 100 + 46, load=0.7, tol=1e-10, glm_tol=1e-8, cpu_sample=12, burst=256),
}
TOL = 1e-8
METRIC = "sec/call (1e7-obs 3-FE OLS)"


def make_data(cfg):
    """Synthetic panel with the configuration's shapes and value distributions (seeded)."""
    n_ind, years, n_firm, k = cfg["n_ind"], cfg["years"], cfg["n_firm"], cfg["k"]
    n = n_ind * years
    rng = np.random.default_rng(cfg["seed"])
    i = np.arange(n)
    ind = (i // years).astype(np.uint32)
    year = (i % years).astype(np.uint32)
    alpha = rng.standard_normal(n_ind)
    gamma = rng.normal(0.0, np.sqrt(0.5), years)
    rows = np.empty((n, 1 + k))
    y = alpha[ind] + gamma[year] + rng.standard_normal(n)
    codes, g = [ind], [n_ind]
    if n_firm:
        firm = (i % n_firm).astype(np.uint32)
        psi = rng.standard_normal(n_firm)
        y += psi[firm]
        codes.append(firm)
        g.append(n_firm)
        for j in range(k):
            x = 0.3 * psi[firm] + np.sqrt(1 - 0.09) * rng.standard_normal(n)
            rows[:, 1 + j] = x
            y += x / (j + 1)
    else:
        for j in range(k):
            x = rng.standard_normal(n)
            rows[:, 1 + j] = x
            y += 1.0 * x
    codes.append(year)
    g.append(years)
    rows[:, 0] = y
    return codes, g, rows


def make_boot_data(cfg):
    """Synthetic C3 panel: firms drawn at random (seeded), y = 0 x1 + effects + noise."""
    n_ind, years, n_firm = cfg["n_ind"], cfg["years"], cfg["n_firm"]
    n = n_ind * years
    rng = np.random.default_rng(cfg["seed"])
    i = np.arange(n)
    ind = (i // years).astype(np.uint32)
    year = (i % years).astype(np.uint32)
    firm = rng.integers(0, n_firm, n).astype(np.uint32)
    _, firm = np.unique(firm, return_inverse=True)
    firm = firm.astype(np.uint32)
    x1 = rng.standard_normal(n)
    y = rng.standard_normal(n_ind)[ind] + rng.normal(0.0, np.sqrt(0.5), years)[year] + \
        rng.standard_normal(n_firm)[firm] + rng.standard_normal(n)
    rows = np.column_stack([y, x1])
    return [ind, year, firm], [n_ind, years, int(firm.max()) + 1], firm, rows


def make_gravity_data(cfg):
    """Synthetic C4 gravity panel (seeded numpy): rows ordered pair-major; FE codes
    exporter#year, importer#year, pair; y ~ Poisson(exp(0.5 x1 - 0.2 log dist + effects + c)) with
    c set so that about 40% of y are 0; effects ~ N(0, 0.5^2)."""
    C, T, S = cfg["countries"], cfg["years"], cfg["sectors"]
    rng = np.random.default_rng(cfg["seed"])
    ex, im = np.meshgrid(np.arange(C), np.arange(C), indexing="ij")
    off = ex != im
    ex, im = ex[off], im[off]
    P = len(ex)
    pair = np.repeat(np.arange(P), T * S)
    year = np.tile(np.repeat(np.arange(T), S), P)
    e_i, i_i = ex[pair], im[pair]
    ey = (e_i * T + year).astype(np.uint32)
    iy = (i_i * T + year).astype(np.uint32)
    n = len(pair)
    ldist = rng.uniform(np.log(100.0), np.log(2e4), P)[pair]
    x1 = rng.standard_normal(n)
    lin = 0.5 * x1 - 0.2 * ldist + rng.normal(0, 0.5, C * T)[ey] + rng.normal(0, 0.5, C * T)[iy] + \
        rng.normal(0, 0.5, P)[pair]
    # intercept for ~40% zeros: P(y = 0) = mean exp(-exp(lin + c))
    lo, hi = -20.0, 20.0
    for _ in range(60):
        c = 0.5 * (lo + hi)
        if np.mean(np.exp(-np.exp(lin + c))) > cfg["zero_share"]:
            lo = c
        else:
            hi = c
    y = rng.poisson(np.exp(lin + c)).astype(float)
    for codes in (ey, iy, pair):  # no FE group may be all zero (the `fe` separation rule)
        assert np.all(np.bincount(codes, weights=y) > 0)
    rows = np.column_stack([y, x1, ldist])
    return [ey, iy, pair.astype(np.uint32)], [C * T, C * T, P], rows


GLM_METRIC = "sec/call (Poisson PML, n=9.95e6, exporter#year + importer#year + pair, robust SEs)"


def run_glm(args, cfg, rank, world, local, pg):
    """C4: one PPML IRLS call per step (seconds per call). Every call, timed or not, runs on a
    fresh session (prepared outside the timed events), so no preconditioner, hierarchy or IRLS
    state of an earlier call carries over."""
    codes, g, rows = make_gravity_data(cfg)
    n = rows.shape[0]
    if args.impl == "reference":
        if rank != 0:
            return
        cpu, _ = glm_cpu_irls(codes, g, rows)
        v = cpu["value"]
        line = {"impl": "reference", "metric": GLM_METRIC, "value": v, "unit": "s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": {"workload": "c4", "n": n},
                "cpu_baseline": cpu,
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch

    import fereg_b200 as fb

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    t0 = time.perf_counter()
    sess = fb.Session(codes, g)
    prepare_s = time.perf_counter() - t0
    order = sess.row_order()
    info = sess.info()
    sess.close()
    rows = np.ascontiguousarray(rows[order])
    prec = fb.PREC_F64 if args.precision == "f64" else fb.PREC_F32_REFINED
    src = torch.from_numpy(rows).to(device)
    pinned = torch.empty(rows.shape, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    np.copyto(host, rows)
    phases, launches, stats = {}, 0, {}

    def step(on_device, profile=False, count=False):
        nonlocal launches
        s = fb.Session(codes, g)  # fresh state (outside the events)
        stream = torch.cuda.ExternalStream(s.stream(), device=device)
        torch.cuda.synchronize(device)
        if profile:
            s.set_profiling(True)
        l0 = s.launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = s.poisson(src.data_ptr() if on_device else host, vce="robust", tol=1e-8, precision=prec,
                        on_device=on_device, nx=2)
        e1.record(stream)
        e1.synchronize()
        if count:
            launches += s.launches() - l0
            for k_, v_ in s.solver_stats().items():
                stats[k_] = stats.get(k_, 0) + v_
        if profile:
            for k, (ms, c) in s.phase_times().items():
                a = phases.get(k, (0.0, 0))
                phases[k] = (a[0] + ms, a[1] + c)
        s.close()
        return e0.elapsed_time(e1) / 1e3, res

    for _ in range(args.warmup):
        step(True)
    barrier(pg)
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            dt, res = step(True, count=True)
            times.append(dt)
    for _ in range(args.prof_steps):
        step(True, profile=True)
    step_s = max_over_ranks(float(np.mean(times)), pg, device)
    e2e = None
    if not args.no_e2e:
        e2e = max_over_ranks(float(np.mean([step(False)[0] for _ in range(2)])), pg, device) / world
    if rank == 0:
        cpu = parity = None
        if not args.no_cpu_baseline and world == 1:
            cpu, ref = glm_cpu_irls(codes, g, make_gravity_data(cfg)[2])
            parity = parity_of(res["b"], res["V"], ref[0], ref[1])
            parity["oracle"] = "oracle/glm.py irls_absorbed at tol 1e-8, inner tolerance down to 1e-10"
        line = {"metric": GLM_METRIC, "value": step_s / world, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if prec == fb.PREC_F64 else "f32+f64", "data": "synthetic",
                "config": {"workload": "c4", "n": n, "irls_iterations": res["iterations"],
                           "pcg_iterations": res["pcg_iterations"], "b_x1": float(res["b"][0]),
                           "status": [int(x) for x in res["status"]], "zero_share": float(np.mean(rows[:, 0] == 0)),
                           "prepare_s": prepare_s, "precision": args.precision, "fresh_session_per_call": True,
                           "parallelism": f"replicas x{world}", "solver_stats_timed_calls": stats},
                "phases_ms_per_step": {k: v[0] / args.prof_steps for k, v in phases.items() if v[1]},
                "phases_note": PHASES_NOTE,
                "roofline": roofline_of(info, phases, n, 3, True, 8 if prec == fb.PREC_F64 else 4, "c4"),
                "cpu_baseline": cpu,
                "parity": parity,
                "clocks": clk.summary(),
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": n * 3 * 8, "d2h_bytes_per_step": 96},
                "gpu_launches": launches}
        print(json.dumps(line), flush=True)


SERVE_METRIC = "served p99 latency (s), mixed stream of 2,000 regressions (60% OLS / 20% IV / 20% logit)"
SERVE_NMAX = 5_000_000


class ServePool:
    """Seeded master columns (5e6 rows, pinned host memory) that the requests of the C5 stream
    slice at offsets that are multiples of 10 (one individual = 10 consecutive rows):
    x1..x12, z1, z2 ~ N(0, 1); endog = 0.7 z1 - 0.4 z2 + 0.5 u + N(0, 1) (u the structural error);
    y = sum_j x_j / j + 0.5 endog + u + N(0, 1); ybin ~ Bernoulli(logistic(0.3 x1 - 0.2 x2)) with
    rows 0 and 1 of every individual set to 1 and 0 (no individual without variation, so the
    `fe` separation rule drops nothing)."""

    def __init__(self, seed, pinned=True):
        import torch

        rng = np.random.default_rng(seed)
        n = SERVE_NMAX
        names = ["y", "ybin", "endog", "z1", "z2"] + [f"x{j}" for j in range(1, 13)]
        self.buf = torch.empty((len(names), n), dtype=torch.float64, pin_memory=pinned)
        a = self.buf.numpy()
        self.col = {k: a[i] for i, k in enumerate(names)}
        X = [rng.standard_normal(n) for _ in range(12)]
        for j in range(12):
            self.col[f"x{j + 1}"][:] = X[j]
        self.col["z1"][:] = rng.standard_normal(n)
        self.col["z2"][:] = rng.standard_normal(n)
        u = rng.standard_normal(n)
        self.col["endog"][:] = 0.7 * self.col["z1"] - 0.4 * self.col["z2"] + 0.5 * u + rng.standard_normal(n)
        y = 0.5 * self.col["endog"] + u + rng.standard_normal(n)
        for j in range(12):
            y += X[j] / (j + 1)
        self.col["y"][:] = y
        p = 1 / (1 + np.exp(-(0.3 * X[0] - 0.2 * X[1])))
        yb = (rng.random(n) < p).astype(np.float64)
        yb[0::10] = 1.0
        yb[1::10] = 0.0
        self.col["ybin"][:] = yb


def serve_request_n(i, seed):
    """The row count of request i of the C5 stream (the first draw of serve_request)."""
    rng = np.random.default_rng(seed + i)
    return int(np.exp(rng.uniform(np.log(1e4), np.log(SERVE_NMAX)))) // 10 * 10


def serve_request(i, seed, pool):
    """Request i of the C5 stream (its own seed): n = exp(U(ln 1e4, ln 5e6)) rounded down to whole
    individuals, 1-4 FEs among indiv (n/10), year (10), firm (n/50 levels; random, or cyclic
    firm = row mod levels as in the 1e7 panel), occupation (100 levels, random); model 60% OLS / 20% IV
    (1 endogenous regressor, 2 instruments) / 20% logit; 1-12 regressors; variance iid / robust /
    cluster (on firm, or indiv when the request has no firm). Returns the submit arguments."""
    rng = np.random.default_rng(seed + i)
    n = int(np.exp(rng.uniform(np.log(1e4), np.log(SERVE_NMAX)))) // 10 * 10
    off = int(rng.integers(0, (SERVE_NMAX - n) // 10 + 1)) * 10
    u = rng.random()
    model = "ols" if u < 0.6 else "iv" if u < 0.8 else "logit"
    nfe = int(rng.integers(1, 5))
    k = int(rng.integers(1, 13))
    idx = np.arange(n, dtype=np.uint32)
    ind = idx // 10
    year = idx % 10
    codes, g = [ind], [n // 10]
    firm = None
    if nfe >= 2:
        codes.append(year)
        g.append(10)
    if nfe >= 3:
        F = max(2, n // 50)
        if rng.random() < 0.5:
            firm = idx % F  # cyclic, as in the 1e7 panel: firm = row mod levels
        else:
            firm = rng.integers(0, F, n).astype(np.uint32)
            present = np.bincount(firm, minlength=F) > 0
            remap = (np.cumsum(present) - 1).astype(np.uint32)
            firm = remap[firm]
            F = int(present.sum())
        codes.append(firm.astype(np.uint32))
        g.append(F)
    if nfe >= 4:
        occ = rng.integers(0, 100, n).astype(np.uint32)
        codes.append(occ)
        g.append(100)
    sl = slice(off, off + n)
    c = pool.col
    vce = ["unadjusted", "robust", "cluster"][int(rng.integers(0, 3))]
    if model == "logit":
        vce = {"unadjusted": "oim"}.get(vce, vce)
    clusters, cl_g = [], []
    if vce == "cluster":
        if firm is not None:
            clusters, cl_g = [codes[2]], [g[2]]
        else:
            clusters, cl_g = [ind], [n // 10]
    if model == "iv":
        nx = k - 1
        cols = [c["y"][sl]] + [c[f"x{j}"][sl] for j in range(1, nx + 1)] + [c["endog"][sl], c["z1"][sl], c["z2"][sl]]
        kw = dict(nendog=1, ninst=2)
    elif model == "logit":
        nx = k
        cols = [c["ybin"][sl]] + [c[f"x{j}"][sl] for j in range(1, nx + 1)]
        kw = {}
    else:
        nx = k
        cols = [c["y"][sl]] + [c[f"x{j}"][sl] for j in range(1, nx + 1)]
        kw = {}
    return dict(model=model, codes=codes, g=g, cols=cols, nx=nx, clusters=clusters, cl_g=cl_g, vce=vce, n=n, kw=kw)


def request_tol(r, cfg):
    """Solver tolerance of a request: OLS / IV solves at cfg["tol"]; logit at the reference's
    default deviance tolerance (GlmOptions: tol 1e-8, final inner tolerance 1e-10)."""
    return cfg["glm_tol"] if r["model"] == "logit" else cfg["tol"]


def submit_request(srv, r, cfg):
    import fereg_b200 as fb

    return srv.submit(r["model"], r["codes"], r["g"], r["cols"], r["nx"], clusters=r["clusters"], cl_g=r["cl_g"],
                      vce=r["vce"], tol=request_tol(r, cfg), precision=fb.PREC_F64, **r["kw"])


def run_serve(args, cfg, rank, world, local, pg):
    """C5: a stream of 2,000 regressions with exponential inter-arrival times at ~70% of the
    measured capacity through the serving engine (fereg_server_*); value = p99 latency (submit to
    result) of the whole stream. The capacity is measured first (the warm-up) on 256 requests
    generated and submitted back to back, in rows per second; the stream's request rate is 70% of
    it over the stream's mean request size."""
    nreq = cfg["requests"]
    if args.impl == "reference":
        if rank != 0:
            return
        run_serve_reference(args, cfg, world)
        return
    import torch

    import fereg_b200 as fb

    torch.cuda.set_device(local)
    pool = ServePool(rank_seed(cfg["seed"], rank))
    srv = fb.Server(workers=args.serve_workers)
    tol = cfg["tol"]

    def collect(tickets, out):
        for t in tickets:
            out.append(srv.wait(t))

    # capacity: requests (seeds after the stream's) generated and submitted back to back, as the
    # stream does but without waiting for arrival times; requests per second at full load, with
    # the client's generation competing for the host as it does in the stream
    burst, tk = [], []
    t0 = time.perf_counter()
    for i in range(cfg["burst"]):
        r = serve_request(nreq + 1000 + i, cfg["seed"], pool)
        burst.append({"n": r["n"]})
        tk.append(submit_request(srv, r, cfg))
    res_b = [srv.wait(t) for t in tk]
    burst_s = time.perf_counter() - t0
    assert all(r["rc"] == 0 for r in res_b), [r["msg"] for r in res_b if r["rc"]]
    cap_rows = sum(r["n"] for r in burst) / burst_s
    cap_req = len(burst) / burst_s
    # the offered load in rows per second: 70% of the burst's rows per second, spread over the
    # stream's own request sizes (a request count would carry the burst sample's size mix over)
    mean_rows = float(np.mean([serve_request_n(i, cfg["seed"]) for i in range(nreq)]))
    rate = cfg["load"] * cap_rows / mean_rows  # requests per second
    arrivals = np.cumsum(np.random.default_rng(cfg["seed"] - 1).exponential(1.0 / rate, nreq))
    barrier(pg)
    results, tickets = [], []
    lock = threading.Lock()
    done_list = []
    waiter_q = []
    cv = threading.Condition(lock)

    def waiter():
        i = 0
        while i < nreq:
            with cv:
                while len(waiter_q) <= i:
                    cv.wait()
                t = waiter_q[i]
            done_list.append(srv.wait(t))
            i += 1

    th = threading.Thread(target=waiter)
    th.start()
    rows_total = 0
    mix = {"ols": 0, "iv": 0, "logit": 0}
    late = []
    h2d = d2h = 0
    reqs_meta = []
    sample = []  # (index, request) of the CPU-baseline sample: the first requests with n <= 2e5
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
        for i in range(nreq):
            r = serve_request(i, cfg["seed"], pool)
            reqs_meta.append({"model": r["model"], "n": r["n"], "nfe": len(r["codes"]), "nx": r["nx"], "vce": r["vce"],
                              "R": len(r["cols"])})
            rows_total += r["n"]
            mix[r["model"]] += 1
            h2d += r["n"] * (8 * len(r["cols"]) + 4 * (len(r["codes"]) + len(r["clusters"])))
            k_all = r["nx"] + (1 if r["model"] == "ols" else 1 if r["model"] == "iv" else 0)
            d2h += 8 * (k_all + k_all * k_all)
            if r["n"] <= 200_000 and len(sample) < cfg["cpu_sample"]:
                sample.append((i, r))
            now = time.perf_counter() - t_start
            if now < arrivals[i]:
                time.sleep(arrivals[i] - now)
            else:
                late.append(now - arrivals[i])
            t = submit_request(srv, r, cfg)
            with cv:
                waiter_q.append(t)
                cv.notify()
        th.join()
        wall = time.perf_counter() - t_start
    res = done_list
    bad = [r for r in res if r["rc"] != 0]
    lat = np.array([r["done_s"] - r["submit_s"] for r in res])
    queue = np.array([r["admit_s"] - r["submit_s"] for r in res])
    first = min(r["submit_s"] for r in res)
    last = max(r["done_s"] for r in res)
    span = last - first
    st = srv.stats()
    p50, p99 = float(np.percentile(lat, 50)), float(np.percentile(lat, 99))
    p99 = max_over_ranks(p99, pg, torch.device("cuda", local))
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = serve_cpu_sample(sample, [res[i] for i, _ in sample], cfg)
    if rank == 0:
        line = {"metric": SERVE_METRIC, "value": p99, "unit": "s", "n_gpus": world, "steps": 1,
                "warmup": 1, "ms_per_step": span * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "c5", "requests": nreq, "mix": mix, "rows_total": rows_total,
                           "offered_rate_req_s": rate, "offered_rows_s": rate * mean_rows, "stream_mean_rows": mean_rows,
                           "load": cfg["load"], "workers": args.serve_workers,
                           "tol": tol, "glm_tol": cfg["glm_tol"], "burst_requests": len(burst),
                           "burst_req_per_s": cap_req, "burst_rows_per_s": cap_rows, "late_submits": len(late),
                           "max_submit_lag_s": float(max(late)) if late else 0.0,
                           "parallelism": f"replicas x{world}", "errors": len(bad),
                           "l2": "inputs of most requests exceed L2; no flush"},
                "p50_s": p50, "p99_s": p99, "mean_queue_s": float(queue.mean()),
                "throughput_req_s": nreq * world / span, "throughput_rows_s": rows_total * world / span,
                "server": st, "clocks": clk.summary(), "gpu_launches": st["launches"],
                "e2e": {"value": p99, "unit": "s", "h2d_bytes_per_step": int(h2d / nreq),
                        "d2h_bytes_per_step": int(d2h / nreq),
                        "note": "a step is one request; host columns in, b and V out, submit to result"}}
        if args.dump:
            with open(args.dump, "w") as f:
                json.dump([{k: x[k] for k in ("submit_s", "admit_s", "done_s", "prep_s", "iterations", "launches")}
                           | r for x, r in zip(res, reqs_meta)], f)
        if cpu is not None:
            line["cpu_baseline"] = cpu["cpu_baseline"]
            line["parity_vs_oracle"] = cpu["parity"]
        print(json.dumps(line), flush=True)
    srv.close()


def oracle_request(r, cfg):
    """The CPU oracle on one request: the session OLS, the 2SLS restatement on the oracle's
    residualized block, or the absorbed logit IRLS. Returns b, V in the server's order."""
    from oracle import glm as oglm
    from oracle import iv as oiv
    from oracle import oracle

    cols = np.column_stack(r["cols"])
    tol = request_tol(r, cfg)
    if r["model"] == "ols":
        sess = oracle.Session(r["codes"], r["g"], r["clusters"], r["cl_g"])
        z = np.ascontiguousarray(cols[sess.row_order()])
        out = sess.ols(z, vce=r["vce"], tol=tol)
        return out["b"], out["V"]
    if r["model"] == "iv":
        Yt = oiv.residualize(r["codes"], r["g"], cols, tol=tol)
        sess = oracle.Session(r["codes"], r["g"], r["clusters"], r["cl_g"])
        df_a = sess.ols(np.ascontiguousarray(cols[sess.row_order()][:, :2]), vce=r["vce"], tol=tol)["scalars"]["df_a"]
        b, V, _, _ = oiv.tsls(Yt, r["nx"], 1, 2, vce=r["vce"], clusters=r["clusters"], df_a=int(df_a))
        return b, V
    cl = (r["clusters"][0], r["cl_g"][0]) if r["clusters"] else None
    b, V, _, _, _ = oglm.irls_absorbed(r["codes"], r["g"], cols[:, 0], cols[:, 1:], "logit", r["vce"], cl, tol=tol)
    return b, V


def serve_cpu_sample(sample, served, cfg):
    """cpu_baseline of C5: the CPU oracle (all host threads) on a bounded sample of the stream's
    requests, one after another; value = the p99 (the maximum, for the sample's size) of their
    service times. The served results of the same requests are compared with the oracle's."""
    from oracle import oracle

    times, errs = [], []
    rows = 0
    for (i, r), s in zip(sample, served):
        t0 = time.perf_counter()
        b, V = oracle_request(r, cfg)
        times.append(time.perf_counter() - t0)
        rows += r["n"]
        kb = len(b)
        se = np.sqrt(np.maximum(np.diag(V), 0.0))
        eb = np.max(np.abs(s["b"][:kb] - b) / np.maximum(np.abs(b), se))
        ev = np.max(np.abs(s["V"][:kb, :kb] - V) / np.max(np.abs(V)))
        errs.append((float(eb), float(ev)))
    return {"cpu_baseline": {"value": float(np.percentile(times, 99)), "unit": "s", "cores": oracle.max_threads(),
                             "kind": "port",
                             "sample": f"{len(sample)} requests of the stream with n <= 2e5 ({rows} rows), each run "
                                       f"alone on the C++ FP64 oracle (session OLS, 2SLS on its residualized block, "
                                       f"absorbed logit IRLS); service time only, no queueing; mean "
                                       f"{float(np.mean(times)):.3f} s, {rows / sum(times):.3g} rows/s"},
            "parity": {"requests": len(errs), "b_err": "|b - b_oracle| / max(|b_oracle|, se_oracle)",
                       "max_rel_err_b": max(e[0] for e in errs),
                       "max_rel_err_V": max(e[1] for e in errs)}}


def run_serve_reference(args, cfg, world):
    """The reference arm of C5: the CPU oracle serves the stream's first requests with n <= 2e5
    one at a time (bounded sample); value = p99 of their service times."""
    pool = ServePool(cfg["seed"], pinned=False)
    sample = []
    i = 0
    while len(sample) < cfg["cpu_sample"]:
        r = serve_request(i, cfg["seed"], pool)
        if r["n"] <= 200_000:
            sample.append(r)
        i += 1
    from oracle import oracle

    times = []
    for r in sample:
        t0 = time.perf_counter()
        oracle_request(r, cfg)
        times.append(time.perf_counter() - t0)
    v = float(np.percentile(times, 99))
    line = {"impl": "reference", "metric": SERVE_METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": 1,
            "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "c5", "requests": len(sample)},
            "cpu_baseline": {"value": v, "unit": "s", "cores": oracle.max_threads(), "kind": "port",
                             "sample": f"the stream's first {len(sample)} requests with n <= 2e5, each alone on the "
                                       f"C++ FP64 oracle; service time, no queueing"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


BOOT_METRIC = "wild-boot reps/s (WCR11, 9,999 Rademacher draws, n=1e6, 3 FE, cluster firm 2e4)"


def boot_cpu_sample(codes, g, rows, rounds=2):
    """The CPU oracle's cost per bootstrap draw: the FE solve of 16 draw columns (the per-draw
    refit's dominant cost), all host threads; the first round is a warm-up."""
    from oracle import oracle

    ab = oracle.Absorber(codes, g)
    rng = np.random.default_rng(1)
    nd = 16
    z = np.ascontiguousarray(rows[ab.row_order(), :1] * rng.choice([-1.0, 1.0], size=(rows.shape[0], nd)))
    times = []
    for _ in range(max(2, rounds)):
        zz = z.copy()
        t0 = time.perf_counter()
        ab.residualize(zz, tol=TOL)
        times.append(time.perf_counter() - t0)
    v = nd / float(np.mean(times[1:]))
    return {"value": v, "unit": "reps/s", "cores": oracle.max_threads(), "kind": "port",
            "sample": f"the FE solve of {nd} draw columns (the per-draw refit's dominant cost), "
                      f"{len(times) - 1} timed rounds, C++ FP64 restatement, all host threads"}


def glm_cpu_irls(codes, g, rows):
    """The CPU oracle's PPML call: the full IRLS of oracle/glm.py (irls_absorbed: the reference's
    loop with the FE solve on the C++ restatement, all host threads, the row work in numpy), robust
    SEs. Returns the cpu_baseline record and (b, V)."""
    from oracle import glm as oglm
    from oracle import oracle

    t0 = time.perf_counter()
    b, V, dev, ll, iters = oglm.irls_absorbed(codes, g, rows[:, 0], rows[:, 1:], "poisson", "robust", tol=1e-8)
    v = time.perf_counter() - t0
    return ({"value": v, "unit": "s", "cores": oracle.max_threads(), "kind": "port",
             "sample": f"one full PPML IRLS call on the full workload ({iters} iterations; FE solves on the C++ "
                       f"FP64 restatement with all host threads, row work in numpy)"}, (b, V))


def roofline_of(sess, phases, n, R, weighted, s_v, workload):
    """Roofline of the dominant timed phase: algorithmic bytes of one call of it (phase_bytes with
    R columns) over its average duration, against the measured copy bandwidth. `sess` is a
    session or its info() dict."""
    hbm, peak_kind = peaks()
    info = sess if isinstance(sess, dict) else sess.info()
    algo = phase_bytes(info, n, R, weighted, s_v)
    timed = {k: v for k, v in phases.items() if k in algo and v[1]}
    if not timed:  # no profiled calls (--prof-steps 0)
        return None
    dom = max(timed, key=lambda k: timed[k][0])
    ms, cnt = timed[dom]
    achieved = algo[dom] / (ms / cnt / 1e3) / 1e9
    kern = phase_kernel(dom, info, n, R)
    return {"bound": "hbm", "kernel": kern, "phase": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": traffic_from_profiles(kern, workload), "traffic_source": TRAFFIC_SOURCE,
            "peak_kind": peak_kind,
            "algorithmic_bytes": algo[dom], "columns": R}


def run_boot(args, cfg, rank, world, local, pg):
    """C3: one WCR11 bootstrap call per step; value = draws per second of the whole job."""
    if args.impl == "reference":
        if rank != 0:
            return
        codes, g, firm, rows = make_boot_data(cfg)
        cpu = boot_cpu_sample(codes, g, rows, 1 + max(1, args.steps // 3))
        v = cpu["value"]
        line = {"impl": "reference", "metric": BOOT_METRIC, "value": v, "unit": "reps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "c3", "n": rows.shape[0], "reps": cfg["reps"]},
                "cpu_baseline": cpu,
                "e2e": {"value": v, "unit": "reps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch

    import fereg_b200 as fb

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    codes, g, firm, rows = make_boot_data(cfg)
    n = rows.shape[0]
    t0 = time.perf_counter()
    sess = fb.Session(codes, g, [firm], [g[2]])
    prepare_s = time.perf_counter() - t0
    rows = np.ascontiguousarray(rows[sess.row_order()])
    prec = fb.PREC_F64 if args.precision == "f64" else fb.PREC_F32_REFINED
    stream = torch.cuda.ExternalStream(sess.stream(), device=device)
    src = torch.from_numpy(rows).to(device)
    work = torch.empty_like(src)
    reps = cfg["reps"]

    def step(on_device):
        if on_device:
            work.copy_(src)
            torch.cuda.synchronize(device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = sess.wildboot(work.data_ptr() if on_device else rows, coef=0, reps=reps, seed=1, tile=args.boot_tile,
                            tol=TOL, boot_precision=prec, on_device=on_device, nx=1)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, res

    for _ in range(args.warmup):
        step(True)
    barrier(pg)
    l0 = sess.launches()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            dt, res = step(True)
            times.append(dt)
    launches = sess.launches() - l0
    phases = profiled_phases(sess, lambda: step(True), args)
    step_s = max_over_ranks(float(np.mean(times)), pg, device)
    e2e = None
    if not args.no_e2e:
        et = [step(False)[0] for _ in range(2)]
        e2e = world * reps / max_over_ranks(float(np.mean(et)), pg, device)
    if rank == 0:
        line = {"metric": BOOT_METRIC, "value": world * reps / step_s, "unit": "reps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == fb.PREC_F64 else "f32+f64",
                "data": "synthetic",
                "config": {"workload": "c3", "n": n, "reps": int(res["reps"]), "tile": args.boot_tile,
                           "precision": args.precision, "prepare_s": prepare_s, "stat": res["stat"],
                           "pvalue": res["pvalue"], "parallelism": f"replicas x{world}"},
                "phases_ms_per_step": {k: v[0] / args.prof_steps for k, v in phases.items() if v[1]},
                "phases_note": PHASES_NOTE,
                # per apply / residualize call of one draw tile (tile columns); the fit's 2-column
                # solve is counted at the tile's width
                "roofline": roofline_of(sess, phases, n, args.boot_tile, False, 8 if prec == fb.PREC_F64 else 4, "c3"),
                "cpu_baseline": None if args.no_cpu_baseline or world > 1 else boot_cpu_sample(codes, g, rows),
                "clocks": clk.summary(),
                "e2e": {"value": e2e, "unit": "reps/s", "h2d_bytes_per_step": n * 2 * 8,
                        "d2h_bytes_per_step": int(res["reps"]) * 8 + 64},
                "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    sess.close()


PHASES_NOTE = ("per-phase CUDA events from --prof-steps extra calls after the timed ones, the same kernels "
               "launched one by one (the timed calls run the PCG iterations as captured graphs)")


def profiled_phases(sess, step, args):
    """Phase times (ms, launches) of args.prof_steps calls with the session's per-phase CUDA events:
    the same kernels, with the PCG iterations launched one by one instead of as graphs."""
    sess.set_profiling(True)
    for _ in range(args.prof_steps):
        step()
    phases = sess.phase_times()
    sess.set_profiling(False)
    return phases


def workload_name(cfg_name):
    if cfg_name == "c2":
        return "OLS y~x1..x10 | indiv(1e6)+firm(1e5, row mod 1e5)+year(10), n=1e7, iid SEs"
    if cfg_name == "c2d":
        return "OLS y~x1..x10 | indiv(1e6)+firm(43478, row mod 43478: connected ring)+year(10), n=1e7, iid SEs"
    if cfg_name == "c2p":
        return "OLS y~x1..x10 | indiv(3e5)+firm(3e4, row mod 3e4)+year(10), n=3e6, iid SEs (profiling case)"
    return "OLS y~x1 | indiv(1e4)+year(10), n=1e5, iid SEs"


PARITY_TOL = 1e-14  # the oracle's solver tolerance for the parity figures (the fixtures' tolerance)
PARITY_TARGET = 1e-8


def parity_of(b, V, b_ref, V_ref):
    """Largest relative error of the coefficients and of the standard errors against the oracle's
    (|b - b_oracle| / |b_oracle|, |se - se_oracle| / se_oracle)."""
    b, b_ref = np.asarray(b), np.asarray(b_ref)
    se = np.sqrt(np.maximum(np.diag(V), 0.0))
    se_ref = np.sqrt(np.maximum(np.diag(V_ref), 0.0))
    kept = np.flatnonzero(se_ref > 0)  # regressors the oracle omits (absorbed, collinear) have se 0
    eb = float(np.max(np.abs(b[kept] - b_ref[kept]) / np.abs(b_ref[kept])))
    es = float(np.max(np.abs(se[kept] - se_ref[kept]) / se_ref[kept]))
    omitted_agree = bool(np.all(se[se_ref == 0] == 0))
    return {"b_max_rel": eb, "se_max_rel": es, "target": PARITY_TARGET, "compared": int(len(kept)),
            "omitted_agree": omitted_agree,
            "ok": bool(eb <= PARITY_TARGET and es <= PARITY_TARGET and omitted_agree)}


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: through NVML every 5 ms
    (so that a timed region of a few tens of milliseconds still holds several samples), else
    nvidia-smi every 200 ms. Read-only queries; no GPU setting is changed."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()
        self.thread = None
        self.lines = []
        self.samples = []  # (sm MHz, max MHz, set of reasons)

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            idx = torch.cuda._get_nvml_device_index(self.device)
        except Exception:
            idx = self.device
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
        except Exception:
            self.nvml = None
        if self.nvml:
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nvml
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        while True:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(smax), {n for n, b in zip(self.NAMES, bits) if r & b}))
            except Exception:
                pass
            if self.stop.wait(0.005):
                break

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.nvml:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        for a, b, rs in self.samples:
            sm.append(a)
            smax = b
            reasons |= rs
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_from_profiles(kernel, workload):
    """Per-launch DRAM bytes (read + write) of `kernel` on `workload` from the committed ncu
    summary profiles/dram_traffic.txt (lines: kernel workload bytes [capture note]): a figure of
    the capture named there, not of this run. None when the kernel has no line."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        with open(path) as f:
            for ln in f:
                parts = ln.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
                    return float(parts[2])
    except OSError:
        pass
    return None


TRAFFIC_SOURCE = "profiles/dram_traffic.txt: one ncu capture per kernel (the file names the capture), not this run"


def phase_bytes(info, n, R, weighted, s_v=8):
    """Algorithmic (compulsory) DRAM bytes of one call of each timed phase.

    M cells, nb blocks (ns of them small), g1 FE1 levels, m reduced coordinates, E = M (nb - ns)
    coordinate-list entries. Gathers that stay in L2 (P, t rows) count once."""
    M, nb, g1, m = info["ncells"], info["nb"], info["g1"], info["m"]
    ns = info["small_blocks"]
    E = M * (nb - ns)
    wrow = n * 8 if weighted else 0
    wcell = M * 8 if weighted else 0
    return {
        "rhs_seg": n * R * 8 + wrow + g1 * R * 8 + g1 * 4 + g1 * 8 + M * ns * 4,
        "rhs_pull": E * 8 + E * R * 8 + g1 * R * 8 + g1 * 8 + m * R * 8,
        "apply_seg": M * nb * 4 + wcell + g1 * 8 + g1 * 4 + g1 * R * s_v + m * R * s_v,
        "apply_pull": E * nb * 4 + g1 * R * s_v + 2 * m * R * s_v + m * 12,
        "residualize": 2 * n * R * 8 + M * nb * 4 + g1 * R * 8 + g1 * 8 + g1 * 4 + m * R * 8,
        "colstats": n * R * 8 + wrow,
        "gram": n * R * 8 + wrow,
        "variance": n * R * 8 + n * 8 + wrow,
    }


PHASE_KERNEL = {"rhs_seg": "k_grhs", "rhs_pull": "k_wpull_rhs", "apply_seg": "k_vseg_apply",
                "apply_pull": "k_vpull_apply", "residualize": "k_wresid", "colstats": "k_colstats_bulk",
                "gram": "k_outer_mma_bulk", "variance": "k_resid_e"}


def phase_kernel(phase, info, n, R):
    """The kernel of a phase: the residualization runs as k_fresid when every cell holds one row
    and the rows have at most 16 columns (the absorber's FR_MAXR)."""
    if phase == "residualize" and info["ncells"] == n and R <= 16:
        return "k_fresid"
    return PHASE_KERNEL[phase]


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        # NCCL on the GPU box; gloo (FEREG_DIST_BACKEND=gloo) for host-only runs of the same logic
        dist.init_process_group(os.environ.get("FEREG_DIST_BACKEND", "nccl"),
                                timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(x, pg, device):
    """The max of x over the ranks (the step time of a multi-GPU run); host tensors under gloo."""
    if pg is None:
        return x
    import torch

    if pg.get_backend() == "gloo":
        device = None
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def rank_seed(seed, rank):
    """Seed of rank `rank`'s replica: each rank serves its own seeded stream (weak scaling)."""
    return seed + 7919 * rank


def barrier(pg):
    if pg is not None:
        pg.barrier()


def oracle_session(codes, g, rows):
    from oracle import oracle

    t0 = time.perf_counter()
    sess = oracle.Session(codes, g)
    prep = time.perf_counter() - t0
    return sess, np.ascontiguousarray(rows[sess.row_order()]), prep


def run_reference(args, cfg_name, cfg, rank, world):
    """The reference's session OLS on the host cores (the CPU oracle), same metric and unit."""
    if rank != 0:
        return
    from oracle import oracle

    codes, g, rows = make_data(cfg)
    sess, rows_ro, prep = oracle_session(codes, g, rows)
    times = []
    for it in range(args.warmup + args.steps):
        z = rows_ro.copy()
        t0 = time.perf_counter()
        sess.ols(z, tol=TOL)
        t1 = time.perf_counter()
        if it >= args.warmup:
            times.append(t1 - t0)
    v = float(np.mean(times))
    threads = oracle.max_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(cfg_name), "n": len(rows), "R": rows.shape[1], "prepare_s": prep},
        "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port",
                         "sample": "one OLS call on the full workload per step (C++ FP64 restatement of the "
                                   "reference's session OLS, OpenMP, all host threads)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=list(CONFIGS))
    ap.add_argument("--precision", default="f64", choices=["f64", "f32r"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle parity figures (profiling runs)")
    ap.add_argument("--prof-steps", type=int, default=3, help="extra calls with per-phase timing (after the timed ones)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer timing (profiling runs)")
    ap.add_argument("--boot-tile", type=int, default=512, help="draws per block-PCG tile (c3)")
    ap.add_argument("--serve-workers", type=int, default=8, help="requests in flight (c5)")
    ap.add_argument("--requests", type=int, default=0, help="stream length override (c5)")
    ap.add_argument("--dump", default="", help="write per-request timings to this file (c5)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    cfg = dict(CONFIGS[args.config])
    if args.requests:
        cfg["requests"] = args.requests
    rank, world, local, pg = dist_setup()
    if args.config in ("c3", "c4", "c5"):
        {"c3": run_boot, "c4": run_glm, "c5": run_serve}[args.config](args, cfg, rank, world, local, pg)
        if pg is not None:
            barrier(pg)
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, args.config, cfg, rank, world)
        if pg is not None:
            pg.destroy_process_group()
        return

    import torch

    import fereg_b200 as fb

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    prec = fb.PREC_F64 if args.precision == "f64" else fb.PREC_F32_REFINED
    codes, g, rows = make_data(cfg)
    n, R = rows.shape
    nx = R - 1
    t0 = time.perf_counter()
    sess = fb.Session(codes, g)
    prepare_s = time.perf_counter() - t0
    info = sess.info()
    rows = np.ascontiguousarray(rows[sess.row_order()])  # the caller hands rows in the session's row order
    stream = torch.cuda.ExternalStream(sess.stream(), device=device)
    src = torch.from_numpy(rows).to(device)
    work = torch.empty_like(src)

    def step_device():
        work.copy_(src)  # fresh inputs each step (outside the timed events)
        torch.cuda.synchronize(device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = sess.ols_device(work.data_ptr(), nx, tol=TOL, precision=prec)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, res

    for _ in range(args.warmup):
        step_device()
    barrier(pg)
    torch.cuda.synchronize(device)
    l0 = sess.launches()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            dt, res = step_device()
            times.append(dt)
    torch.cuda.synchronize(device)
    barrier(pg)
    launches = sess.launches() - l0
    step_s = max_over_ranks(float(np.mean(times)), pg, device)
    value = step_s / world
    phases = profiled_phases(sess, step_device, args)
    # a second session of the same data: the preparation without the process's one-time set-up
    # (library load, CUDA context)
    t0 = time.perf_counter()
    sess2 = fb.Session(codes, g)
    prepare_warm_s = time.perf_counter() - t0
    sess2.close()

    # e2e: the same call through the C ABI with the block in pinned host memory
    pinned = torch.empty((n, R), dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    np.copyto(host, rows)

    def step_e2e():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sess.ols(host, tol=TOL, precision=prec)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    e2e_s = None
    if not args.no_e2e:
        for _ in range(2):
            step_e2e()
        barrier(pg)
        e2e_times = [step_e2e() for _ in range(max(3, args.steps // 2))]
        e2e_s = max_over_ranks(float(np.mean(e2e_times)), pg, device) / world
    k_all = nx + 1
    d2h = (k_all + k_all * k_all + nx) * 8

    # roofline of the dominant kernel phase (largest share of the timed phases)
    hbm, peak_kind = peaks()
    algo = phase_bytes(info, n, R, False, 8 if prec == fb.PREC_F64 else 4)
    timed = {k: v for k, v in phases.items() if k in algo and v[1]}
    dom = max(timed, key=lambda k: timed[k][0]) if timed else None  # none without profiled calls
    if dom:
        ms, cnt = timed[dom]
        achieved = algo[dom] / (ms / cnt / 1e3) / 1e9
        kern = phase_kernel(dom, info, n, R)
        traffic = traffic_from_profiles(kern, args.config)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle

        osess, orows, oprep = oracle_session(codes, g, make_data(cfg)[2])
        ts = []
        for _ in range(2):
            z = orows.copy()
            t1 = time.perf_counter()
            osess.ols(z, tol=TOL)
            ts.append(time.perf_counter() - t1)
        cpu = {"value": float(np.mean(ts)), "unit": "s", "cores": oracle.max_threads(), "kind": "port",
               "sample": "2 OLS calls on the full workload (C++ FP64 restatement of the reference's session OLS, "
                         f"OpenMP); its session prepare took {oprep:.3f} s"}
    parity = None
    if rank == 0 and world == 1 and not args.no_parity:
        # the oracle's answer at the fixtures' tolerance on the same rows (untimed): the error of
        # every coefficient and standard error of the last timed call
        from oracle import oracle

        osess, orows, _ = oracle_session(codes, g, make_data(cfg)[2])
        ref = osess.ols(orows, tol=PARITY_TOL, maxiter=100000)
        parity = parity_of(res["b"], res["V"], ref["b"], ref["V"])
        parity["oracle_tol"] = PARITY_TOL
        parity["k"] = len(ref["b"])
        osess.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == fb.PREC_F64 else "f32+f64", "data": "synthetic",
            "config": {"workload": workload_name(args.config), "n": n, "R": R, "cells": info["ncells"],
                       "m": info["m"], "g1": info["g1"], "pcg_iterations": int(res["scalars"]["ic"]), "tol": TOL,
                       "precision": args.precision, "l2": "inputs (880 MB) larger than L2, no flush",
                       "parallelism": f"replicas x{world}", "prepare_s": prepare_s, "prepare_warm_s": prepare_warm_s,
                       "b_x1": float(res["b"][0]), "solver_stats": sess.solver_stats()},
            "roofline": {"bound": "hbm", "kernel": kern, "phase": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic, "traffic_source": TRAFFIC_SOURCE,
                         "peak_kind": peak_kind,
                         "algorithmic_bytes": algo[dom]} if dom else None,
            "phases_ms_per_step": {k: v[0] / max(1, args.prof_steps) for k, v in phases.items() if v[1]},
            "phases_note": PHASES_NOTE,
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clk.summary(),
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": n * R * 8, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    sess.close()
    if pg is not None:
        barrier(pg)
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
