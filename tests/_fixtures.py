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
