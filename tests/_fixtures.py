"""Loaders for the committed reghdfe fixtures (tests/golden/)."""

import csv
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FACTORS = ["id", "year", "firm", "region", "c1", "c2"]


def load_data():
    with open(os.path.join(GOLDEN, "ols_data.csv")) as f:
        rows = list(csv.DictReader(f))
    return {k: np.array([float(r[k]) for r in rows]) for k in rows[0]}


def load_fixtures():
    with open(os.path.join(GOLDEN, "ols_fixtures.json")) as f:
        return json.load(f)


def nums(v):
    return np.array([np.nan if x is None else float(x) for x in v])


def model_args(spec, data):
    """Arguments of an OLS call (oracle.ols / fereg_b200.ols) for a fixture spec."""
    fidx = {f: i for i, f in enumerate(FACTORS)}
    factors = [data[f] for f in FACTORS]
    absorb = [[fidx[f] for f in t] for t in spec["absorb"]]
    clusters = [[fidx[c]] for c in spec["vce"]]
    vce = "cluster" if spec["vce"] else ("robust" if spec["robust"] else "unadjusted")
    return dict(
        factors=factors, absorb=absorb, y=data[spec["y"]], x=[data[x] for x in spec["x"]], clusters=clusters,
        weights=data[spec["weight"]] if spec["weight"] else None, weight_kind=spec["weight_kind"], vce=vce,
        singletons=spec["singletons"], noconstant=spec["noconstant"], firstpair=spec["firstpair"],
    )


def load_csv(name):
    with open(os.path.join(GOLDEN, name)) as f:
        rows = list(csv.DictReader(f))
    return {k: np.array([float(r[k]) for r in rows]) for k in rows[0]}


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def restrict(codes, alive):
    """Codes of the kept rows, renumbered densely in ascending order, and their count."""
    u, inv = np.unique(codes[alive], return_inverse=True)
    return inv.astype(np.uint32), len(u)


def prepare_iv(spec, data):
    """Sample preparation of an IV fixture as the reference's Session::prepare does it
    (factorize, drop_singletons with fweights, restrict): kept mask, singletons dropped, FE
    terms, cluster dimensions, kept weights."""
    from oracle import oracle

    fac = {f: oracle.factorize(data[f]) for f in ("idcode", "year")}
    terms = [fac[f] for f in spec["absorb"]]
    w = data[spec["weight"]] if spec["weight"] else None
    fw = w if spec["weight_kind"] == "fweight" else None
    alive, nsing = oracle.drop_singletons([c for c, _ in terms], [g for _, g in terms], fw)
    terms = [restrict(c, alive) for c, _ in terms]
    clusters = [restrict(fac[c][0], alive) for c in spec["cluster"]]
    return alive, nsing, terms, clusters, (None if w is None else w[alive])


def iv_block(spec, data, alive):
    cols = [spec["y"]] + spec["exog"] + spec["endog"] + spec["inst"]
    return np.ascontiguousarray(np.stack([data[c][alive] for c in cols], axis=1))


def load_poisson():
    """The committed ppmlhdfe fixtures and their data sets (tests/golden/make_golden.py)."""
    data = {name: load_csv(f"glm_{name}.csv") for name in ("gravity", "auto", "problem1")}
    return load_json("poisson_fixtures.json"), data


def _interact(parts):
    """Dense codes (ascending) of the interaction of factor codes, with the level count."""
    key = np.zeros(len(parts[0][0]), dtype=np.uint64)
    for codes, g in parts:
        key = key * np.uint64(g) + codes.astype(np.uint64)
    u, inv = np.unique(key, return_inverse=True)
    return inv.astype(np.uint32), len(u)


def prepare_poisson(spec, data):
    """Sample preparation of a Poisson fixture as Session::prepare does it for ppmlhdfe: the
    rows of the fixture's `if` condition, factorize, interactions, then cyclically the singleton
    drops (unless singletons are kept) and the `fe` rule (sample.rs:74: rows of an FE group whose
    y sums to 0) until neither changes the sample, then restrict. ppmlhdfe reports both kinds of
    drops as singletons. Returns the kept mask over all input rows, the rows dropped, the kept
    terms, the cluster dimensions and the kept n x (1 + k) block [y, x...] in kept order."""
    from oracle import oracle

    n_all = len(data[spec["y"]])
    base = np.ones(n_all, dtype=bool)
    base[[i - 1 for i in spec["exclude"]]] = False
    names = sorted({f for t in spec["absorb"] for f in t} | {f for t in spec["cluster"] for f in t})
    fac = {f: oracle.factorize(data[f][base]) for f in names}
    terms = [_interact([fac[f] for f in t]) for t in spec["absorb"]]
    y_all = data[spec["y"]][base]
    alive = np.ones(int(base.sum()), dtype=bool)
    while True:
        before = int(alive.sum())
        if not spec["keepsing"]:
            idx = np.flatnonzero(alive)
            a2, _ = oracle.drop_singletons([restrict(c, alive)[0] for c, _ in terms],
                                           [restrict(c, alive)[1] for c, _ in terms], None)
            alive[idx[~a2]] = False
        for c, g in terms:
            s = np.bincount(c[alive], weights=y_all[alive], minlength=g)
            alive &= s[c] > 0
        if int(alive.sum()) == before:
            break
    nsing = int(base.sum()) - int(alive.sum())
    terms = [restrict(c, alive) for c, _ in terms]
    cl = [restrict(_interact([fac[f] for f in t])[0], alive) for t in spec["cluster"]]
    y = y_all[alive]
    block = np.ascontiguousarray(np.column_stack([y] + [data[x][base][alive] for x in spec["x"]]))
    keep = np.zeros(n_all, dtype=bool)
    keep[np.flatnonzero(base)[alive]] = True
    return keep, nsing, terms, cl, block


def load_separation():
    """The committed ppmlhdfe fixtures fitted with sep(fe relu) and their data sets."""
    fx = load_json("separation_fixtures.json")
    data = {f["spec"]["data"]: load_csv(f"glm_{f['spec']['data']}.csv") for f in fx}
    return fx, data


def prepare_separation(spec, data, check, drop=None):
    """Session::glm_separate's rounds (glm/mod.rs:454-505) for a sep(fe relu) fixture: the rows
    from `first_obs` on; per round the cyclic singleton drops (unless kept) and the `fe` rule
    until stable (`drop(codes, g, y, keepsing) -> alive`, the oracle's by default), then the
    separation check `check(terms, block) -> separated rows (kept order)` on the kept sample;
    separated rows leave and the next round prepares the rest, until a check finds none. A
    no-absorb fixture absorbs the constant (one term with one level). Returns the kept mask over
    all rows, the separated and the singleton counts, the kept terms and the [y, x...] block."""
    n_all = len(data[spec["y"]])
    base = np.zeros(n_all, dtype=bool)
    base[spec["first_obs"]:] = True
    y_all = data[spec["y"]][base]
    from oracle import oracle

    if spec["absorb"]:
        fac = {f: oracle.factorize(data[f][base]) for t in spec["absorb"] for f in t}
        terms0 = [_interact([fac[f] for f in t]) if len(t) > 1 else fac[t[0]] for t in spec["absorb"]]
    else:
        terms0 = [(np.zeros(int(base.sum()), dtype=np.uint32), 1)]
    X_all = np.column_stack([data[x][base] for x in spec["x"]]) if spec["x"] else np.zeros((int(base.sum()), 0))

    def oracle_drop(codes, g, y, keepsing):
        alive = np.ones(len(y), dtype=bool)
        while True:
            before = int(alive.sum())
            if not keepsing:
                idx = np.flatnonzero(alive)
                a2, _ = oracle.drop_singletons([restrict(c, alive)[0] for c in codes],
                                               [restrict(c, alive)[1] for c in codes], None)
                alive[idx[~a2]] = False
            for c, gq in zip(codes, g):
                s = np.bincount(c[alive], weights=y[alive], minlength=gq)
                alive &= s[c] > 0
            if int(alive.sum()) == before:
                return alive

    drop = drop or oracle_drop
    alive = np.ones(int(base.sum()), dtype=bool)
    nsep = nsing = 0
    while True:
        idx = np.flatnonzero(alive)
        a2 = drop([c[idx] for c, _ in terms0], [g for _, g in terms0], y_all[idx], spec["keepsing"])
        nsing += int((~a2).sum())
        alive[idx[~a2]] = False
        idx = np.flatnonzero(alive)
        terms = [restrict(c, alive) for c, _ in terms0]
        block = np.ascontiguousarray(np.column_stack([y_all[idx], X_all[idx]]))
        sep = check(terms, block)
        if not sep.any():
            break
        nsep += int(sep.sum())
        alive[idx[sep]] = False
    keep = np.zeros(n_all, dtype=bool)
    keep[np.flatnonzero(base)[alive]] = True
    return keep, nsep, nsing, terms, block
