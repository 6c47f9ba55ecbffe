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
