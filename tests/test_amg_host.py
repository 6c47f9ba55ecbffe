"""The multigrid hierarchy of an escalated block, built on the host (no GPU): every level is a
graph Laplacian (zero row sums, the constants in its null space), the levels shrink, and the
coarsest level is small enough for the dense grounded factor (at most 384 nodes)."""

import numpy as np

import fereg_b200 as fb


def ring(n_ind, F, years=10):
    i = np.arange(n_ind * years)
    return [(i // years).astype(np.uint32), (i % F).astype(np.uint32)], [n_ind, F]


def test_ring_hierarchy_is_a_laplacian_at_every_level():
    codes, g = ring(40000, 7997)
    h = fb.amg_probe(codes, g)
    assert h["levels"] >= 2 and h["sizes"][0] == 7997
    assert all(a > b for a, b in zip(h["sizes"], h["sizes"][1:]))
    assert h["sizes"][-1] <= 384
    assert np.all(h["row_sum"] <= 1e-10)


def test_random_graph_hierarchy():
    rng = np.random.default_rng(3)
    n_ind, years, F = 20000, 5, 3000
    n = n_ind * years
    firm = rng.integers(0, F, n).astype(np.uint32)
    codes = [np.repeat(np.arange(n_ind), years).astype(np.uint32), firm]
    h = fb.amg_probe(codes, [n_ind, F])
    assert h["levels"] >= 2 and h["sizes"][-1] <= 384 and np.all(h["row_sum"] <= 1e-10)


def test_small_structure_has_no_hierarchy():
    codes, g = ring(100, 97)
    assert fb.amg_probe(codes, g)["levels"] == 0
