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


def _joint_problem(n=10, PL=3, seed=7):
    rng = np.random.default_rng(seed)
    P = PL + 1
    H, g = np.zeros((n, P, P)), rng.normal(size=(n, P))
    for i in range(n):
        J = rng.normal(size=(12, P))
        H[i] = J.T @ J
    free = np.ones((n, PL))
    free[::3, 1] = 0.0                                # some voxels hold a value
    return H, g, free


def _schur_worker(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    import bmc_oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        H, g, free = _joint_problem()
        mine = np.arange(rank, H.shape[0], world)    # this rank's voxels
        Y, w, sums = O.schur_partial(H[mine], g[mine], free[mine], 0.05, 1)
        t = torch.tensor(sums, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)     # the one collective of a sharded step: four numbers
        d, ds = O.schur_back(Y, w, t.numpy(), 0.05, 1)
        for k, i in enumerate(mine):
            for j in range(d.shape[1]):
                out[i * d.shape[1] + j] = d[k, j]
        out[len(out) - 1 - rank] = ds
    finally:
        dist.destroy_process_group()


def test_sharded_joint_step_equals_the_dense_solve():
    """fit_joint_uneven over several ranks: each shard eliminates its voxels, the four Schur sums are
    all-reduced, and every rank back-substitutes -- the dense damped step of the whole problem."""
    import bmc_oracle as O
    H, g, free = _joint_problem()
    n, PL = free.shape
    ctx = mp.get_context("spawn")
    out = ctx.Array("d", n * PL + 2)
    port = _free_port()
    procs = [ctx.Process(target=_schur_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    d_want, ds_want = O.joint_step_dense(H, g, free, 0.05, 1)
    got = np.array(out[:n * PL]).reshape(n, PL)
    np.testing.assert_allclose(got, d_want, rtol=1e-10, atol=1e-12)
    assert out[n * PL] == out[n * PL + 1] == __import__("pytest").approx(ds_want, rel=1e-10)
    assert (got[free == 0] == 0).all()
