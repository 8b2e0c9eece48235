"""The benchmark's multi-rank logic on CPU (gloo, world size 2): the reported step time is the
slowest rank's, and every rank simulates its own voxels. No GPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                       # rank 1 is the slow one
        out[rank] = bench.max_over_ranks(ms)
        P, _ = bench.voxel_params(16, 4, seed=bench.rank_seed(rank))
        out[2 + rank] = float(P[3, 0])               # first k of the first voxel
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_ranks_and_ranks_own_their_voxels():
    ctx = mp.get_context("spawn")
    out = ctx.Array("d", 4)
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 15.0
    assert out[2] != out[3]


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
