"""bench.py's JSON line on the host: the reference arm (the CPU oracle) on the small C1 workload
prints one line with the keys of the bench contract."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "c1",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is False
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert "workload" in d["config"] and d["warmup"] >= 3


def test_phase_kernel_names_the_residualization_kernel():
    """The roofline's kernel: the pipelined row-order residualization when every cell holds one
    row and the rows have at most 16 columns, the warp-tile kernel otherwise."""
    sys.path.insert(0, ROOT)
    import bench

    one_row = {"ncells": 1000}
    assert bench.phase_kernel("residualize", one_row, 1000, 11) == "k_fresid"
    assert bench.phase_kernel("residualize", one_row, 1000, 17) == "k_wresid"
    assert bench.phase_kernel("residualize", {"ncells": 900}, 1000, 11) == "k_wresid"
    assert bench.phase_kernel("apply_pull", one_row, 1000, 11) == "k_vpull_apply"


def test_serve_request_sizes_match_the_stream():
    """The C5 offered load uses the stream's request sizes, computed without building the
    requests: each equals the size serve_request draws."""
    sys.path.insert(0, ROOT)
    import bench

    class Pool:  # the columns are sliced, not read, for the size
        col = {k: __import__("numpy").zeros(bench.SERVE_NMAX) for k in
               ["y", "ybin", "endog", "z1", "z2"] + [f"x{j}" for j in range(1, 13)]}

    seed = bench.CONFIGS["c5"]["seed"]
    pool = Pool()
    for i in (0, 1, 7, 123):
        assert bench.serve_request_n(i, seed) == bench.serve_request(i, seed, pool)["n"]
