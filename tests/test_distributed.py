"""Multi-rank logic on CPU (gloo, world size 2), no GPU: the benchmark's step time is the slowest rank's
and every rank simulates its own voxels; the sharded joint fit's step sequence -- the product's own LM
loop (bmc_b200.uneven._joint_lm) with voxels split over two ranks -- takes the steps of one rank holding
every voxel and of the oracle's dense joint LM."""
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


# ------------------------------------------------------------------------------------------------
# the product's joint LM loop over two ranks
# ------------------------------------------------------------------------------------------------
T_GRID = np.linspace(0.0, 3.0, 9)


def _toy(n=8, seed=3):
    """Per voxel amplitude and rate, one shared rate offset: y_i(t) = A_i exp(-(k_i + s) t), noisy data."""
    rng = np.random.default_rng(seed)
    A, k = rng.uniform(0.5, 2.0, n), rng.uniform(0.2, 1.5, n)
    s_true = 0.3
    y = A[:, None] * np.exp(-(k[:, None] + s_true) * T_GRID[None, :])
    return y + 0.01 * rng.standard_normal(y.shape)


class _CpuSteps:
    """The local arithmetic of one rank for the toy model, on the CPU (what _JointSteps does on the GPU):
    normal equations per voxel, the oracle's Schur elimination and back-substitution, trial costs."""

    def __init__(self, data, free):
        import torch
        self.torch, self.data, self.free = torch, data, free

    def _model(self, x_loc, x_s):
        A, k = x_loc[:, 0].numpy()[:, None], x_loc[:, 1].numpy()[:, None]
        e = np.exp(-(k + x_s.numpy()[0]) * T_GRID[None, :])
        return A * e, e

    def normal(self, x_loc, x_s, moved=None):
        if moved is None or bool(moved[0]):
            y, e = self._model(x_loc, x_s)
            r = y - self.data
            dA, dk = e, -T_GRID[None, :] * y
            J = np.stack([dA, dk, dk], axis=-1)                 # d/dA, d/dk, d/ds (ds = dk)
            J[:, :, :2] *= self.free[:, None, :]
            self.H = np.einsum("ntp,ntq->npq", J, J)
            self.g = np.einsum("ntp,nt->np", J, r)
            self.c = (r * r).sum()
        return self.torch.tensor([self.c], dtype=self.torch.float64)

    def eliminate(self, lam):
        import bmc_oracle as O
        self.Y, self.w, sums = O.schur_partial(self.H, self.g, self.free, float(lam[0]), 1)
        return self.torch.tensor(sums, dtype=self.torch.float64)

    def back(self, sums, lam):
        import bmc_oracle as O
        d, ds = O.schur_back(self.Y, self.w, sums.numpy(), float(lam[0]), 1)
        return self.torch.tensor(d), self.torch.tensor([ds], dtype=self.torch.float64)

    def costs(self, x_loc, x_s):
        y, _ = self._model(x_loc, x_s)
        return self.torch.tensor(((y - self.data) ** 2).sum(axis=1))


def _toy_fit(data, free, ranks_of=None, allsum=None, n_iter=8):
    import torch
    from bmc_b200.uneven import _joint_lm
    n = data.shape[0]
    mine = np.arange(n) if ranks_of is None else ranks_of
    steps = _CpuSteps(data[mine], free[mine])
    x_loc = torch.tensor(np.tile([1.0, 0.8], (mine.size, 1)), dtype=torch.float64)
    x_s = torch.tensor([0.1], dtype=torch.float64)
    lo_l, hi_l = torch.tensor([0.0, 0.0], dtype=torch.float64), torch.tensor([5.0, 5.0], dtype=torch.float64)
    lo_s, hi_s = torch.tensor([0.0], dtype=torch.float64), torch.tensor([2.0], dtype=torch.float64)
    return _joint_lm(steps, x_loc, x_s, lo_l, hi_l, lo_s, hi_s, 1e-2, n_iter, allsum)


def _lm_worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        data = _toy()
        free = np.ones((data.shape[0], 2))
        free[2, 1] = 0.0                                  # one voxel holds its rate
        mine = np.arange(rank, data.shape[0], world)

        def allsum(t):
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            return t
        x_loc, x_s, costs = _toy_fit(data, free, mine, allsum)
        for k, i in enumerate(mine):
            out[2 * i], out[2 * i + 1] = float(x_loc[k, 0]), float(x_loc[k, 1])
        n = data.shape[0]
        out[2 * n + rank] = float(x_s[0])
        out[2 * n + 2 + rank] = float(costs[-1])
    finally:
        dist.destroy_process_group()


def test_sharded_joint_lm_takes_the_one_rank_and_dense_steps():
    """Two gloo ranks run the product's joint LM loop on their own voxels (Schur sums and costs
    all-reduced): the same iterates as one rank with every voxel and as the oracle's dense joint LM."""
    import bmc_oracle as O
    data = _toy()
    n = data.shape[0]
    free = np.ones((n, 2))
    free[2, 1] = 0.0
    ctx = mp.get_context("spawn")
    out = ctx.Array("d", 2 * n + 4)
    port = _free_port()
    procs = [ctx.Process(target=_lm_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = np.array(out[:2 * n]).reshape(n, 2)
    assert out[2 * n] == out[2 * n + 1] and out[2 * n + 2] == out[2 * n + 3]   # the ranks agree
    x1, s1, c1 = _toy_fit(data, free)                                            # one rank, every voxel
    # (the sums of two shards add in another order than one rank's: ~1e-10 after 8 steps)
    np.testing.assert_allclose(got, x1.numpy(), rtol=1e-8)
    assert out[2 * n] == __import__("pytest").approx(float(s1[0]), rel=1e-8)
    assert out[2 * n + 2] == __import__("pytest").approx(float(c1[-1]), rel=1e-8)

    # the dense oracle LM over [A_i, k_i] + [s], the held rate fixed by the free mask
    fr = np.concatenate([free.ravel(), [1.0]])

    def resid_jac(x, need_jac=True):
        A, k, s_ = x[:-1:2], x[1:-1:2], x[-1]
        e = np.exp(-(k[:, None] + s_) * T_GRID[None, :])
        y = A[:, None] * e
        J = np.zeros((n * T_GRID.size, 2 * n + 1))
        for i in range(n):
            rows = slice(i * T_GRID.size, (i + 1) * T_GRID.size)
            J[rows, 2 * i] = e[i]
            J[rows, 2 * i + 1] = -T_GRID * y[i]
            J[rows, -1] = -T_GRID * y[i]
        return (y - data).ravel(), J
    x0 = np.concatenate([np.tile([1.0, 0.8], n), [0.1]])
    lo = np.concatenate([np.zeros(2 * n), [0.0]])
    hi = np.concatenate([np.full(2 * n, 5.0), [2.0]])
    xo = O.levenberg_marquardt(resid_jac, x0, lo, hi, n_iter=8, free=fr)
    np.testing.assert_allclose(got, xo[:-1].reshape(n, 2), rtol=1e-8)
    assert out[2 * n] == __import__("pytest").approx(xo[-1], rel=1e-8)
