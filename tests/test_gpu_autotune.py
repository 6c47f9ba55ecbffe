"""The S*P autotuner (absorber.cu autotune_apply): every grid it may choose gives the same bits,
so a tuned solve equals the default-grid solve (FEREG_AUTOTUNE=0) exactly, FP64 and FP32-refined,
on a panel above the tuning threshold (2^20 cells)."""

import os

import numpy as np
import pytest

import bench
import fereg_b200 as fb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [fb.PREC_F64, fb.PREC_F32_REFINED])
def test_tuned_solve_is_bit_identical(precision):
    codes, g, rows = bench.make_data(dict(n_ind=110_000, years=10, n_firm=4_783, k=3, seed=21))
    out = []
    for tune in ("0", "1"):
        os.environ["FEREG_AUTOTUNE"] = tune
        try:
            ab = fb.Absorber(codes, g)
            z = np.ascontiguousarray(rows[ab.row_order()])
            res = ab.residualize(z, tol=1e-10, precision=precision)
            out.append((z, res["iterations"]))
            ab.close()
        finally:
            os.environ.pop("FEREG_AUTOTUNE", None)
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])
