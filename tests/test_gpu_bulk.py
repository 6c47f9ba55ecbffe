"""The row passes that stream a contiguous block through shared memory by TMA bulk copies (column
statistics, the weighted Gram) agree with the register-load passes. The bulk path runs when the
block starts on a 16-byte boundary and holds at least 128 x 592 rows; the same block one double
off that boundary takes the register-load path. Same session, same data: coefficients and
variances agree to 1e-10 (only the order of the sums differs)."""
import numpy as np
import pytest

import fereg_b200 as fb
from tests._gen import panel


@pytest.mark.gpu
@pytest.mark.parametrize("vce", ["unadjusted", "robust", "cluster"])
def test_bulk_row_passes_match_register_loads(vce):
    import torch

    codes, g, w, _ = panel(n_ind=16_000, years=10, n_firm=3_000, seed=31)
    n = len(codes[0])
    assert n >= 128 * 592
    nx = 10
    rng = np.random.default_rng(32)
    X = rng.standard_normal((n, nx))
    y = X @ (1.0 / np.arange(1, nx + 1)) + rng.standard_normal(n)
    clusters = [codes[2]] if vce == "cluster" else []
    cl_g = [g[2]] if vce == "cluster" else []
    sess = fb.Session(codes, g, clusters=clusters, cl_g=cl_g)
    rows = np.ascontiguousarray(np.column_stack([y, X])[sess.row_order()])
    r = rows.shape[1]
    src = torch.from_numpy(rows.ravel()).to("cuda")
    buf = torch.empty(n * r + 2, dtype=torch.float64, device="cuda")  # base on a 256-byte boundary
    out = {}
    for off in (0, 1):  # 0: 16-byte aligned (bulk copies); 1: 8 bytes off (register loads)
        view = buf[off:off + n * r]
        view.copy_(src)
        assert (view.data_ptr() % 16 == 0) == (off == 0)
        out[off] = sess.ols_device(view.data_ptr(), nx, vce=vce)
    b0, b1 = np.asarray(out[0]["b"]), np.asarray(out[1]["b"])
    V0, V1 = np.asarray(out[0]["V"]), np.asarray(out[1]["V"])
    assert np.max(np.abs(b0 - b1)) <= 1e-10 * np.max(np.abs(b0))
    assert np.max(np.abs(V0 - V1)) <= 1e-10 * np.max(np.abs(V0))
    for key in ("rss", "tss", "r2", "N", "df_a"):
        a, b = out[0]["scalars"][key], out[1]["scalars"][key]
        assert abs(a - b) <= 1e-10 * max(1.0, abs(a))
