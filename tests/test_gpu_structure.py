"""The cell structure built on the device (fereg_structure_compare) against the host build,
element for element (structure.rs:356-527): the row order, seg_off, cell_row, coord and the
coordinate-sorted lists (offsets, cells, segments, other-block coordinates), with the FE1 choice,
the block classification and the small-block work.

Every panel of the parity tests runs twice: as generated (rows already in key order for most) and
with its rows shuffled, which makes the device sort them.
"""

import numpy as np
import pytest

import bench
import fereg_b200 as fb
from tests._gen import panel
from tests.test_gpu_parity import CASES

pytestmark = pytest.mark.gpu


def panels():
    for name, spec in CASES.items():
        codes, g, _, _ = panel(**spec)
        if name == "one_fe":
            codes, g = codes[:1], g[:1]
        yield name, codes, g
    codes, g, _ = bench.make_data(dict(n_ind=100_000, years=10, n_firm=10_000, k=1, seed=3))
    yield "cyclic_1e6", codes, g
    codes, g, _ = bench.make_gravity_data(dict(countries=60, years=20, sectors=3, seed=5, zero_share=0.4))
    yield "gravity", codes, g


PANELS = list(panels())


@pytest.mark.parametrize("shuffle", [False, True])
@pytest.mark.parametrize("name,codes,g", PANELS, ids=[p[0] for p in PANELS])
def test_device_structure_is_the_host_structure(name, codes, g, shuffle):
    if shuffle:
        perm = np.random.default_rng(17).permutation(len(codes[0]))
        codes = [np.ascontiguousarray(c[perm]) for c in codes]
    diff = fb.structure_compare(codes, g)
    assert all(v == 0 for v in diff.values()), (name, shuffle, diff)
