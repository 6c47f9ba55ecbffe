"""The oracle's PCG path checked by the properties that define the projection.

e = z - D(D'WD)^+ D'W z is the unique vector with (1) D'W e = 0 (W-orthogonal to every level
dummy of every term) and (2) z - e in span(D), here z - e = fit_rows(coefs) (the reference's
DenseAbsorber oracle, reference.rs:1-6, states the same projection through an explicit SVD).
"""

import numpy as np
import pytest

from oracle import oracle
from tests._gen import panel
from tests.test_gpu_parity import CASES, build


def orthogonality(codes, g, w, e):
    """max over terms and levels of |sum_level w e| relative to sum |w e|."""
    we = e if w is None else w * e
    scale = np.abs(we).sum() + 1e-300
    worst = 0.0
    for c, gq in zip(codes, g):
        s = np.bincount(c, weights=we, minlength=gq)
        worst = max(worst, float(np.max(np.abs(s))) / scale)
    return worst


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_projection_properties(case):
    codes, g, w, z = build(case)
    orc = oracle.Absorber(codes, g, w)
    pi = orc.row_order()
    zr = z.copy()
    info = orc.residualize(zr, tol=1e-13, maxiter=200000, want_coefs=True)
    w_rows = None if w is None else w[pi]
    codes_rows = [c[pi] for c in codes]
    for j in range(z.shape[1]):
        assert orthogonality(codes_rows, g, w_rows, zr[:, j]) <= 1e-9, (case, j)
        fit = orc.fit_rows(info["coefs"], j)
        assert np.max(np.abs(z[:, j] - fit - zr[:, j])) <= 1e-9 * max(1.0, np.max(np.abs(z[:, j])))
