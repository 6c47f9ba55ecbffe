"""Parity of the B200 absorber (through the C ABI) with the CPU oracle on seeded panels.

Integer work (row order, cell structure, redundant coordinates) must match exactly; floating
point within the stated tolerances: operator pieces 1e-12 relative (same FP64 math, different
summation order), residualized columns 1e-9 relative to the column scale at tol 1e-12.
"""

import numpy as np
import pytest

import fereg_b200 as fb
from oracle import oracle
from tests._gen import panel

pytestmark = pytest.mark.gpu

CASES = {
    "two_fe": dict(n_ind=600, years=10),
    "three_fe_random": dict(n_ind=6000, years=10, n_firm=5000, seed=1),
    "three_fe_weighted": dict(n_ind=5000, years=10, n_firm=4500, seed=2, weighted=True),
    "repeated_cells": dict(n_ind=1500, years=6, n_firm=5000, seed=3, repeat=3),
    "dense_small": dict(n_ind=6000, years=10, n_firm=900, seed=10),
    "ring": dict(n_ind=6000, years=10, n_firm=4603, firm="cyclic", seed=4),
    "disconnected": dict(n_ind=7000, years=8, n_firm=6000, seed=5, disconnected=True),
    "unbalanced": dict(n_ind=7000, years=10, n_firm=5200, seed=6, drop=0.2, weighted=True),
    "small_firms": dict(n_ind=500, years=10, n_firm=300, seed=7),
    "nested": dict(n_ind=5000, years=10, n_firm=4200, firm="nested", seed=8),
    "one_fe": dict(n_ind=400, years=5, seed=9),
    # 160 rows per individual with random firms: FE1 levels of ~160 cells, split across tiles
    "long_segments": dict(n_ind=5000, years=10, n_firm=4500, seed=11, repeat=16, weighted=True),
    # six terms: five blocks behind FE1, more than the warp tiles stage in shared memory
    "six_fe": dict(n_ind=8000, years=6, n_firm=2000, seed=12, extra=(40, 300, 5000), weighted=True),
}


def build(case):
    spec = dict(CASES[case])
    one_fe = case == "one_fe"
    codes, g, w, z = panel(**spec)
    if one_fe:
        codes, g = codes[:1], g[:1]
    return codes, g, w, z


def rel(a, b):
    scale = max(1.0, float(np.max(np.abs(b)))) if b.size else 1.0
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0


@pytest.fixture(scope="module", params=list(CASES))
def pair(request):
    codes, g, w, z = build(request.param)
    return request.param, fb.Absorber(codes, g, w), oracle.Absorber(codes, g, w), z


def test_structure_and_weights_match(pair):
    _, gpu, orc, _ = pair
    assert (gpu.m, gpu.g1, gpu.ncells, gpu.nb, gpu.m_small, gpu.fe1) == (orc.m, orc.g1, orc.ncells, orc.nb, orc.m_small, orc.fe1)
    assert np.array_equal(gpu.row_order(), orc.row_order())
    a, b = gpu.weight_state(), orc.weight_state()
    assert np.array_equal(a["redundant"], b["redundant"])
    for k in ("n1", "nr", "diag"):
        assert rel(a[k], b[k]) <= 1e-12, k
    assert abs(a["sw"] - b["sw"]) <= 1e-12 * b["sw"]


def test_operator_pieces_match(pair):
    _, gpu, orc, z = pair
    if gpu.m == 0:
        pytest.skip("no reduced system")
    rng = np.random.default_rng(11)
    p = rng.standard_normal((gpu.m, 3))
    assert rel(gpu.apply(p), orc.apply(p)) <= 1e-12
    y1, b11, q1, s1 = gpu.rhs(z)
    y2, b12, q2, s2 = orc.rhs(z)
    assert rel(y1, y2) <= 1e-12 and rel(b11, b12) <= 1e-12
    assert rel(q1, q2) <= 1e-12 and rel(s1, s2) <= 1e-12
    if gpu.m_small <= 1024:  # beyond it the device keeps Jacobi on the small block
        assert rel(gpu.precond(p), orc.precond(p)) <= 1e-10


def test_residualize_matches_oracle(pair):
    name, gpu, orc, z = pair
    z1, z2 = z.copy(), z.copy()
    i1 = gpu.residualize(z1, tol=1e-12, maxiter=100000, want_coefs=True)
    i2 = orc.residualize(z2, tol=1e-12, maxiter=100000, want_coefs=True)
    for j in range(z.shape[1]):
        assert rel(z1[:, j], z2[:, j]) <= 1e-9, (name, j)
    if gpu.m_small <= 1024:  # beyond it the device keeps Jacobi on the small block
        assert i1["exact"] == i2["exact"]
    # the coefficients reproduce the projection: z - fit = residual
    for j in range(z.shape[1]):
        fit = gpu.fit_rows(i1["coefs"], j)
        assert rel(z[:, j] - fit, z1[:, j]) <= 1e-9
    # normalized FE values are unique (solve.rs:1319-1343)
    if gpu.fe1 >= 0:
        tv1 = gpu.term_values(i1["coefs"], 0)
        tv2 = orc.term_values(i2["coefs"], 0)
        for a, b in zip(tv1, tv2):
            assert rel(a, b) <= 1e-7


@pytest.mark.parametrize("r", [1, 11, 17, 40])
@pytest.mark.parametrize("weighted", [False, True])
def test_residualize_one_row_per_cell(r, weighted):
    """One row per cell with FE1 segments of 1 to 40 cells: the pipelined row-order tiles (R 1
    and 11), the warp-tile kernel of wider rows (R 17 and 40, in column chunks), and the CTA tiles
    past 32 cells."""
    rng = np.random.default_rng(40 + r + 100 * weighted)
    n_ind = 2500
    k = rng.integers(1, 41, n_ind)
    ind = np.repeat(np.arange(n_ind), k).astype(np.uint32)
    year = np.concatenate([rng.permutation(41)[:c] for c in k]).astype(np.uint32)
    firm = rng.integers(0, 700, len(ind)).astype(np.uint32)
    codes = [ind, firm, year]
    g = [n_ind, 700, 41]
    w = rng.uniform(0.2, 3.0, len(ind)) if weighted else None
    gpu, orc = fb.Absorber(codes, g, w), oracle.Absorber(codes, g, w)
    assert gpu.ncells == gpu.n
    z = rng.standard_normal((gpu.n, r)) + 0.01 * ind[:, None]
    z1, z2 = z.copy(), z.copy()
    i1 = gpu.residualize(z1, tol=1e-12, maxiter=100000, want_coefs=True)
    orc.residualize(z2, tol=1e-12, maxiter=100000)
    for j in range(r):
        assert rel(z1[:, j], z2[:, j]) <= 1e-9, j
        assert rel(z[:, j] - gpu.fit_rows(i1["coefs"], j), z1[:, j]) <= 1e-9, j


def test_residualize_is_deterministic(pair):
    _, gpu, _, z = pair
    z1, z2 = z.copy(), z.copy()
    gpu.residualize(z1, tol=1e-10)
    gpu.residualize(z2, tol=1e-10)
    assert np.array_equal(z1, z2)


def test_warm_start_and_set_weights(pair):
    name, gpu, orc, z = pair
    rng = np.random.default_rng(5)
    w = rng.uniform(0.5, 2.0, gpu.n)
    gpu.set_weights(w)
    orc.set_weights(w)
    try:
        z1, z2 = z.copy(), z.copy()
        i1 = gpu.residualize(z1, tol=1e-12, maxiter=100000, want_coefs=True)
        orc.residualize(z2, tol=1e-12, maxiter=100000)
        for j in range(z.shape[1]):
            assert rel(z1[:, j], z2[:, j]) <= 1e-9, (name, j)
        # a warm start from the solution converges at once to the same answer
        z3 = z.copy()
        gpu.residualize(z3, tol=1e-12, maxiter=100000, warm=i1["coefs"])
        for j in range(z.shape[1]):
            assert rel(z3[:, j], z1[:, j]) <= 1e-9
        assert np.array_equal(gpu.weights(), w)
    finally:
        gpu.set_weights(None)
        orc.set_weights(None)


def test_bad_weights_rejected(pair):
    _, gpu, _, _ = pair
    w = np.ones(gpu.n)
    w[3] = -1.0
    with pytest.raises(fb.FeregError) as e:
        gpu.set_weights(w)
    assert e.value.rc == 198


def test_maxiter_reports_convergence_error():
    codes, g, w, z = build("ring")
    gpu = fb.Absorber(codes, g, w)
    with pytest.raises(fb.FeregError) as e:
        gpu.residualize(z.copy(), tol=1e-14, maxiter=3)
    assert e.value.rc == 430


def test_refined_fp32_matches_oracle(pair):
    """FP32 PCG iterations inside FP64 refinement reach the FP64 answer (tol 1e-10)."""
    name, gpu, orc, z = pair
    z1, z2 = z.copy(), z.copy()
    i1 = gpu.residualize(z1, tol=1e-10, maxiter=100000, want_coefs=True, precision=fb.PREC_F32_REFINED)
    orc.residualize(z2, tol=1e-12, maxiter=100000)
    for j in range(z.shape[1]):
        assert rel(z1[:, j], z2[:, j]) <= 1e-7, (name, j)
    for j in range(z.shape[1]):
        fit = gpu.fit_rows(i1["coefs"], j)
        assert rel(z[:, j] - fit, z1[:, j]) <= 1e-9


@pytest.mark.parametrize("case", ["three_fe_weighted", "repeated_cells", "small_firms"])
@pytest.mark.parametrize("r", [1, 2, 7, 16, 37])
def test_column_counts_match_oracle(case, r):
    """Column blocks of every padded width (1..32) and blocks wider than one chunk."""
    spec = dict(CASES[case], r=r)
    codes, g, w, z = panel(**spec)
    gpu, orc = fb.Absorber(codes, g, w), oracle.Absorber(codes, g, w)
    z1, z2 = z.copy(), z.copy()
    gpu.residualize(z1, tol=1e-12, maxiter=100000)
    orc.residualize(z2, tol=1e-12, maxiter=100000)
    for j in range(r):
        assert rel(z1[:, j], z2[:, j]) <= 1e-9, (case, r, j)
    y1, b11, q1, s1 = gpu.rhs(z)
    y2, b12, q2, s2 = orc.rhs(z)
    assert rel(y1, y2) <= 1e-12 and rel(b11, b12) <= 1e-12
    assert rel(q1, q2) <= 1e-12 and rel(s1, s2) <= 1e-12


def test_device_weights_match_oracle(pair):
    """set_weights_device (the weight state computed on the device) against the oracle's."""
    import torch

    name, gpu, orc, z = pair
    rng = np.random.default_rng(17)
    w = rng.uniform(0.3, 3.0, gpu.n)
    wd = torch.from_numpy(w).to("cuda")
    gpu.set_weights_device(wd.data_ptr())
    orc.set_weights(w)
    try:
        a, b = gpu.weight_state(), orc.weight_state()
        assert np.array_equal(a["redundant"], b["redundant"]), name
        for key in ("n1", "nr", "diag"):
            assert rel(a[key], b[key]) <= 1e-12, (name, key)
        assert abs(a["sw"] - b["sw"]) <= 1e-12 * b["sw"]
        assert np.array_equal(gpu.weights(), w)
        z1, z2 = z.copy(), z.copy()
        gpu.residualize(z1, tol=1e-12, maxiter=100000)
        orc.residualize(z2, tol=1e-12, maxiter=100000)
        for j in range(z.shape[1]):
            assert rel(z1[:, j], z2[:, j]) <= 1e-9, (name, j)
    finally:
        gpu.set_weights(None)
        orc.set_weights(None)


@pytest.mark.parametrize("case", ["dense_small", "small_firms", "two_fe", "repeated_cells"])
def test_device_small_factor_matches_oracle(case):
    """With weights set on the device, the dense small factor is assembled on the device by rows
    (weights.cuh k_small_rows; dense_small: 910 small coordinates, small_firms 310, two_fe 10);
    the preconditioner matches the oracle's host assembly."""
    import torch

    codes, g, w0, z = build(case)
    gpu = fb.Absorber(codes, g)
    orc = oracle.Absorber(codes, g)
    if gpu.m_small == 0 or gpu.m_small > 1024:
        pytest.skip("no dense small block")
    w = np.random.default_rng(23).uniform(0.3, 3.0, gpu.n)
    gpu.set_weights_device(torch.from_numpy(w).to("cuda").data_ptr())
    orc.set_weights(w)
    p = np.random.default_rng(24).standard_normal((gpu.m, 2))
    assert rel(gpu.precond(p), orc.precond(p)) <= 1e-10
