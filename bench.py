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
    # OLS y ~ x1 | indiv + year, n = 1e4 indiv x 10 years.
    "c1": dict(n_ind=10_000, years=10, n_firm=0, k=1, seed=10**5 * 100 + 42),
    # WCR11 wild cluster bootstrap of b_x1 (H0 true): y ~ x1 | indiv + year + firm, cluster firm,
    # n = 1e5 indiv x 10 years, firm random in 2e4, 9,999 Rademacher draws (seed 1).
    "c3": dict(n_ind=100_000, years=10, n_firm=20_000, k=1, seed=10**6 * 100 + 44, reps=9_999),
    # Poisson PML (gravity): trade ~ x1 + log dist | exporter#year + importer#year + pair, 200
    # countries x 50 years, 39,800 directed pairs x 5 rows (sectors) per pair-year, ~40% zeros,
    # robust SEs.
    "c4": dict(countries=200, years=50, sectors=5, seed=10**7 * 100 + 45, zero_share=0.40),
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
    """C4: one PPML IRLS call per step (seconds per call)."""
    codes, g, rows = make_gravity_data(cfg)
    n = rows.shape[0]
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle

        ab = oracle.Absorber(codes, g)
        rng = np.random.default_rng(1)
        w = rng.uniform(0.5, 2.0, n)
        ab.set_weights(w)
        z = np.ascontiguousarray(rows[ab.row_order()])
        ts = []
        for _ in range(2):
            zz = z.copy()
            t0 = time.perf_counter()
            ab.residualize(zz, tol=1e-8)
            ts.append(time.perf_counter() - t0)
        per_it = float(np.mean(ts))
        iters = 12
        v = per_it * iters
        line = {"impl": "reference", "metric": GLM_METRIC, "value": v, "unit": "s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": {"workload": "c4", "n": n},
                "cpu_baseline": {"value": v, "unit": "s", "cores": oracle.max_threads(), "kind": "port",
                                 "sample": f"one weighted FE solve of [z, x1, ldist] ({per_it:.3f} s, C++ FP64 "
                                           f"restatement, all host threads) times {iters} IRLS iterations"},
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
    rows = np.ascontiguousarray(rows[sess.row_order()])
    prec = fb.PREC_F64 if args.precision == "f64" else fb.PREC_F32_REFINED
    stream = torch.cuda.ExternalStream(sess.stream(), device=device)
    src = torch.from_numpy(rows).to(device)
    pinned = torch.empty(rows.shape, dtype=torch.float64, pin_memory=True)
    host = pinned.numpy()
    np.copyto(host, rows)

    def step(on_device):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = sess.poisson(src.data_ptr() if on_device else host, vce="robust", tol=1e-8, precision=prec,
                           on_device=on_device, nx=2)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, res

    for _ in range(args.warmup):
        step(True)
    barrier(pg)
    sess.set_profiling(True)
    l0 = sess.launches()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            dt, res = step(True)
            times.append(dt)
    launches = sess.launches() - l0
    phases = sess.phase_times()
    sess.set_profiling(False)
    step_s = max_over_ranks(float(np.mean(times)), pg, device)
    e2e = None
    if not args.no_e2e:
        e2e = max_over_ranks(float(np.mean([step(False)[0] for _ in range(2)])), pg, device) / world
    if rank == 0:
        line = {"metric": GLM_METRIC, "value": step_s / world, "unit": "s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if prec == fb.PREC_F64 else "f32+f64", "data": "synthetic",
                "config": {"workload": "c4", "n": n, "irls_iterations": res["iterations"],
                           "pcg_iterations": res["pcg_iterations"], "b_x1": float(res["b"][0]),
                           "status": [int(x) for x in res["status"]], "zero_share": float(np.mean(rows[:, 0] == 0)),
                           "prepare_s": prepare_s, "precision": args.precision,
                           "parallelism": f"replicas x{world}"},
                "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items() if v[1]},
                "clocks": clk.summary(),
                "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": n * 3 * 8, "d2h_bytes_per_step": 96},
                "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    sess.close()


BOOT_METRIC = "wild-boot reps/s (WCR11, 9,999 Rademacher draws, n=1e6, 3 FE, cluster firm 2e4)"


def run_boot(args, cfg, rank, world, local, pg):
    """C3: one WCR11 bootstrap call per step; value = draws per second of the whole job."""
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle

        codes, g, firm, rows = make_boot_data(cfg)
        ab = oracle.Absorber(codes, g)
        rng = np.random.default_rng(1)
        nd = 16
        z = np.ascontiguousarray(rows[ab.row_order(), :1] * rng.choice([-1.0, 1.0], size=(rows.shape[0], nd)))
        times = []
        for it in range(max(1, args.warmup // 3) + max(1, args.steps // 3)):
            zz = z.copy()
            t0 = time.perf_counter()
            ab.residualize(zz, tol=TOL)
            times.append(time.perf_counter() - t0)
        v = nd / float(np.mean(times[1:] if len(times) > 1 else times))
        line = {"impl": "reference", "metric": BOOT_METRIC, "value": v, "unit": "reps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "c3", "n": rows.shape[0], "reps": cfg["reps"]},
                "cpu_baseline": {"value": v, "unit": "reps/s", "cores": oracle.max_threads(), "kind": "port",
                                 "sample": f"the FE solve of {nd} draw columns per step (the per-draw refit's "
                                           "dominant cost), C++ FP64 restatement, all host threads"},
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
    sess.set_profiling(True)
    l0 = sess.launches()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            dt, res = step(True)
            times.append(dt)
    launches = sess.launches() - l0
    phases = sess.phase_times()
    sess.set_profiling(False)
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
                "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items() if v[1]},
                "clocks": clk.summary(),
                "e2e": {"value": e2e, "unit": "reps/s", "h2d_bytes_per_step": n * 2 * 8,
                        "d2h_bytes_per_step": int(res["reps"]) * 8 + 64},
                "gpu_launches": launches}
        print(json.dumps(line), flush=True)
    sess.close()


def workload_name(cfg_name):
    if cfg_name == "c2":
        return "OLS y~x1..x10 | indiv(1e6)+firm(1e5, row mod 1e5)+year(10), n=1e7, iid SEs"
    return "OLS y~x1 | indiv(1e4)+year(10), n=1e5, iid SEs"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


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
    summary profiles/dram_traffic.txt (lines: kernel workload bytes)."""
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


PHASE_KERNEL = {"rhs_seg": "k_wseg_rhs", "rhs_pull": "k_wpull_rhs", "apply_seg": "k_wseg_apply",
                "apply_pull": "k_wpull_apply", "residualize": "k_wresid", "colstats": "k_colstats1",
                "gram": "k_outer_mma", "variance": "k_resid_e"}


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(x, pg, device):
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


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
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer timing (profiling runs)")
    ap.add_argument("--boot-tile", type=int, default=512, help="draws per block-PCG tile (c3)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    cfg = CONFIGS[args.config]
    rank, world, local, pg = dist_setup()
    if args.config in ("c3", "c4"):
        (run_boot if args.config == "c3" else run_glm)(args, cfg, rank, world, local, pg)
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
    sess.set_profiling(True)
    l0 = sess.launches()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            dt, res = step_device()
            times.append(dt)
    torch.cuda.synchronize(device)
    barrier(pg)
    launches = sess.launches() - l0
    phases = sess.phase_times()
    sess.set_profiling(False)
    step_s = max_over_ranks(float(np.mean(times)), pg, device)
    value = step_s / world

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
    dom = max(timed, key=lambda k: timed[k][0])
    ms, cnt = timed[dom]
    achieved = algo[dom] / (ms / cnt / 1e3) / 1e9
    kern = PHASE_KERNEL[dom]
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

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == fb.PREC_F64 else "f32+f64", "data": "synthetic",
            "config": {"workload": workload_name(args.config), "n": n, "R": R, "cells": info["ncells"],
                       "m": info["m"], "g1": info["g1"], "pcg_iterations": int(res["scalars"]["ic"]), "tol": TOL,
                       "precision": args.precision, "l2": "inputs (880 MB) larger than L2, no flush",
                       "parallelism": f"replicas x{world}", "prepare_s": prepare_s,
                       "b_x1": float(res["b"][0])},
            "roofline": {"bound": "hbm", "kernel": kern, "phase": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes": algo[dom]},
            "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items() if v[1]},
            "cpu_baseline": cpu,
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
