"""Seeded synthetic panels for the parity tests (numpy PCG64 seeds fixed per case).

The graph shapes follow the reference's solver integration cases (crates/fereg-core/tests/
solver.rs): random bipartite 2-3 FE, weighted, ring (cyclic firms), repeated cells, disconnected
and nested designs.
"""

import numpy as np


def panel(n_ind=600, years=10, n_firm=None, firm="random", seed=0, weighted=False, repeat=1, r=3,
          disconnected=False, drop=0.0, extra=()):
    rng = np.random.default_rng(seed)
    n = n_ind * years * repeat
    ind = np.repeat(np.arange(n_ind), years * repeat)
    year = np.tile(np.repeat(np.arange(years), repeat), n_ind)
    codes, g = [ind.astype(np.uint32)], [n_ind]
    codes.append(year.astype(np.uint32))
    g.append(years)
    if n_firm:
        if firm == "random":
            f = rng.integers(0, n_firm, n)
        elif firm == "cyclic":
            f = (np.arange(n) // repeat) % n_firm
        elif firm == "nested":  # firm constant within individual
            f = (ind * 7919) % n_firm
        if disconnected:  # two halves of individuals use disjoint firm sets
            half = ind >= n_ind // 2
            f = np.where(half, n_firm // 2 + f % (n_firm - n_firm // 2), f % (n_firm // 2))
        codes.append(f.astype(np.uint32))
        g.append(n_firm)
    for levels in extra:  # further random terms (designs with more than three FE)
        codes.append(rng.integers(0, levels, n).astype(np.uint32))
        g.append(levels)
    keep = np.ones(n, dtype=bool)
    if drop > 0:
        keep = rng.random(n) >= drop
    codes = [c[keep] for c in codes]
    # re-densify codes after drops
    out_codes, out_g = [], []
    for c in codes:
        u, inv = np.unique(c, return_inverse=True)
        out_codes.append(inv.astype(np.uint32))
        out_g.append(len(u))
    n = int(keep.sum())
    w = rng.uniform(0.2, 3.0, n) if weighted else None
    z = rng.standard_normal((n, r))
    z[:, 0] += out_codes[0] * 0.01
    return out_codes, out_g, w, z
