"""The multi-GPU plumbing of bench.py on the host: two ranks over gloo (world size 2, 127.0.0.1).

A run on N GPUs is N independent replicas with no data-path collective: each rank runs its own
seeded workload (here a dry-run serving engine, no GPU), and the only collectives are the barrier
and the max over ranks of the timed value. Checked: every rank gets the global max, the ranks'
seeds differ, and each rank's requests complete on its own server.
"""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), FEREG_DIST_BACKEND="gloo")
    import numpy as np

    import bench
    import fereg_b200 as fb

    r, w, local, pg = bench.dist_setup()
    assert (r, w) == (rank, world)
    srv = fb.Server(workers=2, hbm_budget=1 << 40, dry_run=True)
    codes = [np.zeros(4, dtype=np.uint32)]
    cols = [np.zeros(4)] * 2
    tickets = [srv.submit("ols", codes, [1], cols, 1, n=1000 * (rank + 1), dry_run_us=2000) for _ in range(5)]
    done = [srv.wait(t) for t in tickets]
    local_value = float(rank + 1) * 10.0
    bench.barrier(pg)
    m = bench.max_over_ranks(local_value, pg, None)
    out[rank] = (m, bench.rank_seed(100, rank), sum(d["N"] for d in done), srv.stats()["completed"])
    srv.close()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replicas_over_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(worker, args=(world, free_port(), out), nprocs=world, join=True)
    res = dict(out)
    assert res[0][0] == res[1][0] == 20.0  # max over ranks on every rank
    assert res[0][1] != res[1][1]  # each replica has its own seed
    assert res[0][2] == 5 * 1000 and res[1][2] == 5 * 2000  # each rank served its own requests
    assert res[0][3] == res[1][3] == 5
