"""Sample preparation on the device (fereg_factorize / combine / drop_singletons / restrict)
against the oracle: bit-exact codes, level counts, kept masks and drop counts.

The reference's definitions: factor.rs:38 (codes in ascending value order, -0 = +0, NaN
rejected), :255 (interaction codes in lexicographic order), :281 (renumbering over the kept
rows); sample.rs:44-72 (cyclic passes over the terms until nterms consecutive passes drop
nothing; per pass a level with count 1 drops its rows as singletons, else a level without
variation in the outcome drops them as fe-separated: Poisson no nonzero y, logit none or all).
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import oracle
from tests._fixtures import FACTORS, load_data, load_fixtures

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["small_ints", "wide_ints", "floats", "negative_zero", "constant"])
def test_factorize_matches_oracle(kind):
    rng = np.random.default_rng({"small_ints": 1, "wide_ints": 2, "floats": 3, "negative_zero": 4,
                                 "constant": 5}[kind])
    n = 200_003
    if kind == "small_ints":  # the direct table
        x = rng.integers(-500, 5000, n).astype(float)
    elif kind == "wide_ints":  # integers over a range wider than max(2n, 2^20): the sort
        x = rng.integers(-(1 << 40), 1 << 40, n).astype(float)
        x[::7] = x[3]  # repeated values
    elif kind == "floats":
        x = np.round(rng.standard_normal(n) * 1e3, 2)
    elif kind == "negative_zero":
        x = rng.choice([-0.0, 0.0, -1.5, 2.25, 1e300, -1e-300], n)
    else:
        x = np.full(n, 7.0)
    a, ga = fb.factorize(x)
    b, gb = oracle.factorize(x)
    assert ga == gb and np.array_equal(a, b)


def test_factorize_rejects_missing():
    x = np.arange(10.0)
    x[4] = np.nan
    with pytest.raises(fb.FeregError) as e:
        fb.factorize(x)
    assert e.value.rc == 198


@pytest.mark.parametrize("wide", [False, True])
def test_combine_matches_oracle(wide):
    rng = np.random.default_rng(7)
    n = 150_000
    nl = [70_000, 9_000, 13] if wide else [40, 11, 3]
    parts = [rng.integers(0, g, n).astype(np.uint32) for g in nl]
    a, ga = fb.combine(parts, nl)
    b, gb = oracle.combine(parts, nl)
    assert ga == gb and np.array_equal(a, b)


def panel(seed, n_ind=4000, years=6, n_firm=900):
    rng = np.random.default_rng(seed)
    n = n_ind * years
    ind = np.repeat(np.arange(n_ind), years).astype(np.uint32)
    year = np.tile(np.arange(years), n_ind).astype(np.uint32)
    keep = rng.random(n) < 0.55  # unbalanced: many singletons
    firm = rng.integers(0, n_firm, n).astype(np.uint32)
    codes = [oracle.factorize(c[keep].astype(float)) for c in (ind, year, firm)]
    return codes, rng


@pytest.mark.parametrize("weighted", [False, True])
def test_drop_singletons_matches_oracle(weighted):
    codes, rng = panel(11)
    c, g = [a for a, _ in codes], [b for _, b in codes]
    fw = rng.integers(1, 4, len(c[0])).astype(float) if weighted else None
    alive, s, f = fb.drop_singletons(c, g, fw)
    oalive, od = oracle.drop_singletons(c, g, fw)
    assert np.array_equal(alive, oalive) and s == od and f == 0
    assert s > 0


def fe_rule_restated(codes, g, y, family, fw=None):
    """sample.rs:154-238 pass semantics, restated in numpy (cyclic passes in absorb order)."""
    n = len(codes[0])
    alive = np.ones(n, dtype=bool)
    w = np.ones(n) if fw is None else fw
    nz = (y != 0).astype(float)
    s_tot = f_tot = 0
    remaining, i = len(codes), 0
    while remaining > 0:
        t = i % len(codes)
        i += 1
        c = codes[t]
        cnt = np.bincount(c[alive], weights=w[alive], minlength=g[t])
        pos = np.bincount(c[alive], weights=(w * nz)[alive], minlength=g[t])
        sing = alive & (cnt[c] == 1.0)
        sep = alive & ~sing & ((pos[c] == 0.0) | ((family == "logit") & (pos[c] == cnt[c])))
        alive &= ~(sing | sep)
        s, f = int(sing.sum()), int(sep.sum())
        s_tot += s
        f_tot += f
        remaining = len(codes) - 1 if s + f > 0 else remaining - 1
    return alive, s_tot, f_tot


@pytest.mark.parametrize("family", ["poisson", "logit"])
def test_fe_separation_matches_restatement(family):
    codes, rng = panel(12)
    c, g = [a for a, _ in codes], [b for _, b in codes]
    n = len(c[0])
    if family == "poisson":
        y = rng.poisson(0.4, n).astype(float)
    else:
        y = (rng.random(n) < 0.3).astype(float)
    alive, s, f = fb.drop_singletons(c, g, y=y, family=family)
    ra, rs, rf = fe_rule_restated(c, g, y, family)
    assert np.array_equal(alive, ra) and (s, f) == (rs, rf)
    assert f > 0


def test_restrict_matches_numpy():
    codes, rng = panel(13)
    c, g = [a for a, _ in codes], [b for _, b in codes]
    alive, _, _ = fb.drop_singletons(c, g)
    for col, gg in zip(c, g):
        out, nl = fb.restrict(col, gg, alive)
        u, inv = np.unique(col[alive], return_inverse=True)
        assert nl == len(u) and np.array_equal(out, inv.astype(np.uint32))


def test_prepare_reproduces_the_fixture_samples():
    """The reghdfe fixtures' e(sample) and num_singletons from the device preparation."""
    data = load_data()
    fidx = {f: i for i, f in enumerate(FACTORS)}
    factors = [data[f] for f in FACTORS]
    for fix in load_fixtures():
        spec = fix["spec"]
        if not spec["absorb"] or not spec["singletons"]:
            continue
        fw = data[spec["weight"]] if spec["weight_kind"] == "fweight" else None
        absorb = [[fidx[f] for f in t] for t in spec["absorb"]]
        prep = fb.prepare(factors, absorb, fw=fw)
        assert np.array_equal(prep["alive"].astype(float), np.array(fix["sample"], dtype=float)), spec["name"]
        assert prep["num_singletons"] == fix["scalars"]["num_singletons"], spec["name"]
