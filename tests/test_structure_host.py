"""The host cell structure and coordinate lists (built in parallel) do not depend on the thread
count: the same digest with 1 and with 4 OpenMP threads, on samples large enough for every
parallel path (sorted and unsorted rows, repeated cells)."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import fereg_b200 as fb
n = 400_000
out = {}
for case in ("sorted", "unsorted", "repeated"):
    rng = np.random.default_rng(7)
    idx = np.arange(n, dtype=np.uint32)
    if case == "sorted":
        ind, year = idx // 10, idx % 10
    else:
        ind, year = rng.integers(0, n // 10, n).astype(np.uint32), rng.integers(0, 10, n).astype(np.uint32)
    firm = rng.integers(0, n // 50, n).astype(np.uint32) if case != "repeated" else rng.integers(0, 3, n).astype(np.uint32)
    occ = rng.integers(0, 100, n).astype(np.uint32) if case != "repeated" else np.zeros(n, dtype=np.uint32)
    codes = [ind, year, firm, occ]
    g = [int(c.max()) + 1 for c in codes]
    out[case] = fb.structure_digest(codes, g)
print(json.dumps(out))
"""


def run(threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_structure_digest_is_thread_count_independent():
    one, four = run(1), run(4)
    assert one == four
    assert one["repeated"]["cells"] < 400_000  # repeated (indiv, year, firm, occ) combinations share cells
    assert one["sorted"]["cells"] == 400_000
