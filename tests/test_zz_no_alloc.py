"""The allocation-free right-hand side entry (fereg_absorber_rhs_noalloc) against fereg_absorber_rhs.

The file sorts last, so in a full run it executes after every other test; it also passes alone in
a fresh process. Each case makes two calls in a row through the C ABI and compares both with the
allocating entry point at the tolerance of the other operator pieces (1e-12 relative).
"""

import numpy as np
import pytest

import fereg_b200 as fb
from tests._gen import panel

pytestmark = pytest.mark.gpu

CASES = {
    # short segments on warp tiles, a small block summed in the segment pass, weights
    "three_fe_weighted": dict(n_ind=5000, years=10, n_firm=4500, seed=2, weighted=True),
    # repeated cells (rows per cell > 1)
    "repeated_cells": dict(n_ind=1500, years=6, n_firm=5000, seed=3, repeat=3),
    # segments longer than a warp tile: CTA tiles and slices completed from partials
    "long_segments": dict(n_ind=5000, years=10, n_firm=4500, seed=11, repeat=16, weighted=True),
    # no reduced system (m = 0)
    "one_fe": dict(n_ind=400, years=5, seed=9),
}


def rel(a, b):
    scale = max(1.0, float(np.max(np.abs(b)))) if b.size else 1.0
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0


def build(case):
    codes, g, w, z = panel(**CASES[case])
    if case == "one_fe":
        codes, g = codes[:1], g[:1]
    return fb.Absorber(codes, g, w), z


@pytest.mark.parametrize("case", list(CASES))
def test_rhs_noalloc_matches_rhs_twice(case):
    import torch

    gpu, z = build(case)
    r = z.shape[1]
    y0, b10, wsq0, wsum0 = gpu.rhs(z)
    dev = torch.device("cuda", 0)
    rows = torch.from_numpy(np.ascontiguousarray(z)).to(dev)
    y = torch.empty(max(1, gpu.m * r), dtype=torch.float64, device=dev)
    b1 = torch.empty(gpu.g1 * r, dtype=torch.float64, device=dev)
    cs = torch.empty(3 * r, dtype=torch.float64, device=dev)
    for call in range(2):
        for t in (y, b1, cs):
            t.fill_(float("nan"))  # every output element must be written by the call
        torch.cuda.synchronize(dev)
        free0 = torch.cuda.mem_get_info(dev)[0]
        gpu.rhs_noalloc(rows.data_ptr(), r, y.data_ptr(), b1.data_ptr(), cs.data_ptr())
        torch.cuda.synchronize(dev)
        if call == 1:  # set-up (the scratch address) is done: the call takes no device memory
            assert torch.cuda.mem_get_info(dev)[0] == free0
        yh = y.cpu().numpy()[: gpu.m * r].reshape(gpu.m, r)
        b1h = b1.cpu().numpy().reshape(gpu.g1, r)
        csh = cs.cpu().numpy().reshape(3, r)
        assert rel(yh, y0) <= 1e-12, (case, call)
        assert rel(b1h, b10) <= 1e-12, (case, call)
        assert rel(csh[0], wsq0) <= 1e-12 and rel(csh[1], wsum0) <= 1e-12, (case, call)
        n1 = gpu.weight_state()["n1"]
        assert rel(csh[2], np.sum(b10 ** 2 / n1[:, None], axis=0)) <= 1e-12, (case, call)


def test_rhs_noalloc_rejects_oversized_scratch():
    import torch

    gpu, z = build("three_fe_weighted")
    r = 120  # the small coordinates' partial rows alone exceed the 16 MiB scratch
    dev = torch.device("cuda", 0)
    rows = torch.zeros((gpu.n, r), dtype=torch.float64, device=dev)
    y = torch.empty(gpu.m * r, dtype=torch.float64, device=dev)
    b1 = torch.empty(gpu.g1 * r, dtype=torch.float64, device=dev)
    cs = torch.empty(3 * r, dtype=torch.float64, device=dev)
    with pytest.raises(fb.FeregError) as e:
        gpu.rhs_noalloc(rows.data_ptr(), r, y.data_ptr(), b1.data_ptr(), cs.data_ptr())
    assert e.value.rc == 198
    assert "static scratch" in str(e.value)
