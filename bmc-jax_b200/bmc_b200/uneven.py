"""Uneven batches: voxels with their own pool counts and event tables, simulated and fitted together.

BMC-JAX runs one event table per Experiment (fitting/experiment.py:43-46) and one pool count per
parameter batch, so a mix of models and protocols is one call per shape class there. Here the voxels of
a pool count share one launch whatever their tables (bmc_uneven_* in include/bmc_b200.h); each voxel
gets the result its own class's call gives. `fit_joint_uneven` fits per-voxel values plus at most one
value shared by every voxel (e.g. water T1) with the joint Levenberg-Marquardt of fitting/joint.py:
149-162 -- one damping for the whole problem, the same damped normal equations -- assembled per voxel
on the GPU and solved through the Schur complement of the shared column (bmc_normal_segments,
bmc_schur_eliminate / bmc_schur_back). Every iteration stays on the device: the damping, the costs and
the accept/reject decision are device tensors, and on one GPU an iteration is replayed from a CUDA graph.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from .simulation import n_cest_of, pack_params, state_size

__all__ = ["UnevenBatch", "UnevenFitResult", "fit_joint_uneven"]


def _table_key(ev):
    import hashlib
    h = hashlib.sha1()
    for a in ev:
        a = np.ascontiguousarray(a)
        h.update(str((a.dtype, a.shape)).encode())
        h.update(a.tobytes())
    return h.digest()


class _Plan:
    """The library's plan of one pool count: a set of event tables and the table of every voxel. `run`
    simulates every voxel's chains (canonical order: voxel-major, then the rows of its table) in one
    launch per tangent pass."""

    def __init__(self, nc: int, tables: Sequence, vox_table: np.ndarray, mz: int):
        torch = _lib.torch_cuda()
        self.nc, self.mz = int(nc), int(mz)
        self.vox_table = np.ascontiguousarray(vox_table, np.int32)
        self.n_rows = np.array([np.shape(t.dt)[0] for t in tables], np.int32)
        n_ev = np.array([np.shape(t.dt)[1] for t in tables], np.int32)
        cat = lambda f, dt: np.concatenate([np.asarray(getattr(t, f), dt).reshape(-1) for t in tables])
        dev = [torch.as_tensor(cat("type", np.int32)).cuda()] + \
              [torch.as_tensor(cat(f, np.float64)).cuda() for f in ("dt", "rf_amp", "rf_phase", "rf_freq")] + \
              [torch.as_tensor(cat("adc_idx", np.int32)).cuda()]
        ts = _lib.TableSet(len(tables), self.n_rows.ctypes.data_as(C.POINTER(C.c_int32)),
                           n_ev.ctypes.data_as(C.POINTER(C.c_int32)), _lib.Events(*[x.data_ptr() for x in dev]))
        nv = self.vox_table.size
        self.chain_start = np.zeros(nv + 1, np.int64)
        nch = C.c_int64()
        plan = C.c_void_p()
        _lib.check(_lib.lib().bmc_uneven_create(self.nc, nv, self.vox_table.ctypes.data_as(C.POINTER(C.c_int32)),
                                                C.byref(ts), self.mz, 1, C.byref(plan), C.byref(nch),
                                                self.chain_start.ctypes.data_as(C.POINTER(C.c_int64))))
        self.plan, self.n_chains = plan, int(nch.value)
        self.d_chain_start = torch.as_tensor(self.chain_start).cuda()

    def run(self, params, m0, tangents=None, jz=None, spread=None, z=None, active=None):
        """z [n_chains] (device) for params [n_fields][n_voxels] and m0 [n_voxels][N] (device, float64);
        with tangents, their derivatives into jz [n_tangents][n_chains]; `spread` a _lib.Spread or None.
        `z`: an output buffer to fill (else a new one); `active`: int32 [n_voxels] on the device, voxels
        with 0 skipped (their outputs left as they were)."""
        torch = _lib.torch_cuda()
        if z is None:
            z = torch.empty(self.n_chains, dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().bmc_uneven_simulate(self.plan, _lib.ptr(params), _lib.ptr(m0),
                                                  None if spread is None else C.byref(spread),
                                                  None if tangents is None else C.byref(tangents), _lib.ptr(active),
                                                  _lib.ptr(z), _lib.ptr(jz), _lib.stream_handle()))
        return z

    def __del__(self):
        try:
            if getattr(self, "plan", None) is not None and self.plan.value:
                _lib.lib().bmc_uneven_destroy(self.plan)
                self.plan = C.c_void_p()
        except Exception:
            pass


class _Group:
    """The voxels of one pool count: their packed parameters and start states on the device and the plan
    of their tables."""

    def __init__(self, nc: int, voxels: List[int], experiments):
        torch = _lib.torch_cuda()
        self.nc, self.voxels = nc, np.asarray(voxels, np.int64)
        exps = [experiments[i] for i in voxels]
        mz = int(exps[0].mz_loc)
        if any(int(e.mz_loc) != mz for e in exps):
            raise ValueError(f"voxels with {nc} CEST pools disagree on mz_loc")
        keys, tables, vt = {}, [], []
        by_obj = {}                                   # id -> key: a table object shared by voxels is hashed once
        for e in exps:
            k = by_obj.get(id(e.events))
            if k is None:
                k = by_obj[id(e.events)] = _table_key(e.events)
            if k not in keys:
                keys[k] = len(tables)
                tables.append(e.events)
            vt.append(keys[k])
        self.plan = _Plan(nc, tables, np.asarray(vt, np.int32), mz)
        self.mz, self.chain_start, self.n_chains = mz, self.plan.chain_start, self.plan.n_chains
        self.d_chain_start = self.plan.d_chain_start
        from .simulation import SimParams
        stacked = SimParams(*[np.stack([np.asarray(getattr(e.params, f), np.float64) for e in exps])
                              for f in SimParams._fields])
        self.params = torch.as_tensor(pack_params(stacked, len(voxels))).cuda()
        self.m0 = torch.as_tensor(np.stack([np.asarray(e.m0, np.float64) for e in exps])).cuda()
        self.N = state_size(nc)

    def run(self, params=None, tangents=None, jz=None):
        return self.plan.run(self.params if params is None else params, self.m0, tangents, jz)


class UnevenBatch:
    """Experiments of one voxel each (own params, event table, start state), grouped by pool count."""

    def __init__(self, experiments: Sequence):
        if not experiments:
            raise ValueError("an uneven batch needs at least one experiment")
        for i, e in enumerate(experiments):
            if np.ndim(e.params.water_r1) != 0:
                raise ValueError(f"experiment {i}: one sample per experiment (scalar water_r1)")
        self.experiments = list(experiments)
        by_nc: Dict[int, List[int]] = {}
        for i, e in enumerate(experiments):
            by_nc.setdefault(n_cest_of(e.params), []).append(i)
        self.groups = [_Group(nc, v, experiments) for nc, v in sorted(by_nc.items())]
        self.n = len(experiments)

    def simulate(self) -> List[np.ndarray]:
        """Z of every voxel (its table's rows), in the experiments' order."""
        out: List[Optional[np.ndarray]] = [None] * self.n
        for g in self.groups:
            z = g.run().cpu().numpy()
            for k, v in enumerate(g.voxels):
                out[v] = z[g.chain_start[k]:g.chain_start[k + 1]]
        return out


@dataclass
class UnevenFitResult:
    """x (n, L) physical values of the sample slots (NaN where a slot does not apply to a voxel, e.g. a
    pool it does not have), `shared` the fitted shared value (or None), rms (n,) of each voxel's
    residual, cost (n_iter,) the summed squared residual after each iteration, names of the slots."""
    x: np.ndarray
    shared: Optional[float]
    rms: np.ndarray
    cost: np.ndarray
    names: List[str]
    shared_name: Optional[str]

    def __getitem__(self, name: str) -> np.ndarray:
        return self.x[:, self.names.index(name)]


class _JointSteps:
    """One rank's share of the joint step on the GPU, the arithmetic `_joint_lm` drives: every voxel's
    normal equations at a point, the Schur elimination and back-substitution of the damped step, and the
    voxels' costs at a trial point. All buffers are allocated once; nothing is read back to the host."""

    def __init__(self, batch, spec, z_meas, loc, shr):
        from .fitting import field_row
        torch = _lib.torch_cuda()
        n, PL, S = batch.n, len(loc), len(shr)
        P = PL + S
        self.batch, self.n, self.PL, self.S, self.P = batch, n, PL, S, P
        scl = spec.scales
        self.scl_loc = [float(scl[l]) for l in loc]
        self.scl_s = float(scl[shr[0]]) if S else 0.0
        free = np.zeros((n, PL))
        for g in batch.groups:
            g.rows = []
            for j, l in enumerate(loc):
                sl = spec.slots[l]
                ok = sl.index is None or sl.index < g.nc
                g.rows.append(field_row(sl.field, sl.index, g.nc) if ok else None)
                if ok:
                    free[g.voxels, j] = 1.0
            g.row_s = field_row(spec.slots[shr[0]].field, spec.slots[shr[0]].index, g.nc) if S else None
            for k, v in enumerate(g.voxels):
                zv = np.asarray(z_meas[v], np.float64).reshape(-1)
                if zv.size != g.chain_start[k + 1] - g.chain_start[k]:
                    raise ValueError(f"z_meas[{v}] has {zv.size} points, its table "
                                     f"{g.chain_start[k + 1] - g.chain_start[k]}")
            ng = len(g.voxels)
            g.zm = torch.as_tensor(np.concatenate([np.asarray(z_meas[v], np.float64).reshape(-1)
                                                   for v in g.voxels])).cuda()
            g.idx = torch.as_tensor(g.voxels).cuda()
            g.seg = torch.repeat_interleave(torch.arange(ng, device="cuda"),
                                            torch.as_tensor(np.diff(g.chain_start)).cuda())
            # tangents: the local slots (zero where a slot does not apply) then the shared one
            tg = _lib.Tangents()
            tg.n_tangents = P
            seed = np.zeros((P, ng))
            for j in range(PL):
                tg.field_row[j] = _lib.SEED_NONE if g.rows[j] is None else g.rows[j]
                if g.rows[j] is not None:
                    seed[j] = self.scl_loc[j]
            if S:
                tg.field_row[PL] = g.row_s
                seed[PL] = self.scl_s
            g.seed = torch.as_tensor(seed).cuda()
            tg.d_seed = g.seed.data_ptr()
            tg.d_dm0 = None
            g.tangents = tg
            f64 = dict(dtype=torch.float64, device="cuda")
            g.jz = torch.empty((P, g.n_chains), **f64)
            g.z_n, g.z_t, g.r = (torch.zeros(g.n_chains, **f64) for _ in range(3))
            g.p_n, g.p_t = torch.empty_like(g.params), torch.empty_like(g.params)
            g.act = torch.ones(ng, dtype=torch.int32, device="cuda")
            g.Hg, g.gg, g.cg = torch.empty((ng, P, P), **f64), torch.empty((ng, P), **f64), torch.empty(ng, **f64)
        f64 = dict(dtype=torch.float64, device="cuda")
        self.free = torch.as_tensor(free).cuda()
        self.free_np = free
        self.H, self.g, self.c = torch.empty((n, P, P), **f64), torch.empty((n, P), **f64), torch.empty(n, **f64)
        self.work = torch.empty((2 * PL + 4) * n + 4, **f64)
        self.sums = torch.empty(4, **f64)
        self.d_loc, self.d_s = torch.empty((n, PL), **f64), torch.zeros(1, **f64)
        self.cost_v = torch.empty(n, **f64)
        self.L = _lib.lib()

    def _params_into(self, g, buf, x_loc, x_s):
        buf.copy_(g.params)
        xv = x_loc.index_select(0, g.idx)
        for j, row in enumerate(g.rows):
            if row is not None:
                buf[row].copy_(xv[:, j] * self.scl_loc[j])
        if self.S:
            buf[g.row_s].copy_((x_s * self.scl_s).expand(buf.shape[1]))

    def normal(self, x_loc, x_s, moved=None):
        """Every voxel's J^T J, J^T r and r.r at (x_loc, x_s); returns the (1,) total r.r. With `moved` a
        (1,) bool tensor that is False, the kernels skip every voxel and the normal equations stay those of
        the unchanged point (same J, same r)."""
        torch = _lib.torch_cuda()
        for g in self.batch.groups:
            if moved is not None:
                g.act.copy_(moved.to(torch.int32).expand(g.act.shape[0]))
            self._params_into(g, g.p_n, x_loc, x_s)
            g.plan.run(g.p_n, g.m0, g.tangents, g.jz, z=g.z_n, active=None if moved is None else g.act)
            torch.sub(g.z_n, g.zm, out=g.r)
            _lib.check(self.L.bmc_normal_segments(len(g.voxels), self.P, g.n_chains, _lib.ptr(g.d_chain_start),
                                                  _lib.ptr(g.jz), _lib.ptr(g.r), _lib.ptr(g.Hg), _lib.ptr(g.gg),
                                                  _lib.ptr(g.cg), _lib.stream_handle()))
            self.H.index_copy_(0, g.idx, g.Hg)
            self.g.index_copy_(0, g.idx, g.gg)
            self.c.index_copy_(0, g.idx, g.cg)
        return self.c.sum().reshape(1)

    def eliminate(self, lam):
        """This rank's four Schur sums of the damped step (the damping read from lam on the device)."""
        _lib.check(self.L.bmc_schur_eliminate(self.n, self.PL, self.S, _lib.ptr(self.H), _lib.ptr(self.g),
                                              _lib.ptr(self.free), -1.0, _lib.ptr(lam), _lib.ptr(self.work),
                                              _lib.ptr(self.sums), _lib.stream_handle()))
        return self.sums

    def back(self, sums, lam):
        """(d_loc (n, PL), d_s (1,)) from the sums of every rank."""
        _lib.check(self.L.bmc_schur_back(self.n, self.PL, self.S, _lib.ptr(sums), -1.0, _lib.ptr(lam),
                                         _lib.ptr(self.work), _lib.ptr(self.d_loc), _lib.ptr(self.d_s),
                                         _lib.stream_handle()))
        return self.d_loc, self.d_s

    def costs(self, x_loc, x_s):
        """(n,) r.r of every voxel at (x_loc, x_s)."""
        torch = _lib.torch_cuda()
        for g in self.batch.groups:
            self._params_into(g, g.p_t, x_loc, x_s)
            g.plan.run(g.p_t, g.m0, z=g.z_t)
            rt = g.z_t - g.zm
            self.cost_v.index_copy_(0, g.idx, torch.zeros(len(g.voxels), dtype=torch.float64,
                                                          device="cuda").index_add_(0, g.seg, rt * rt))
        return self.cost_v


def _joint_lm(steps, x_loc, x_s, lo_l, hi_l, lo_s, hi_s, lam0, n_iter, allsum=None, graph=False,
              callback=None):
    """The joint Levenberg-Marquardt of fitting/joint.py:375-416 with the step of joint.py:149-162: one
    damping for the whole problem; the damped step from the Schur sums of every rank; the trial point
    clipped into the bounds; accepted if the summed cost falls (lam x 0.5, the normal equations refreshed
    at the new point), else lam x 3 and the same normal equations again (the same x gives the same J).

    `steps` supplies the local arithmetic (normal, eliminate, back, costs: see _JointSteps); every
    quantity is a torch tensor on the steps' device, and the loop reads no value back to the host
    (unless `callback`, which receives (iteration, cost) as numbers). `allsum(t)` sums a tensor over the
    ranks in place and returns it (None: one rank). `graph`: capture one iteration in a CUDA graph and
    replay it (one rank, no callback). Returns (x_loc, x_s, cost per iteration) as tensors."""
    import torch
    red = allsum if allsum is not None else (lambda t: t)
    dev = x_loc.device
    x_loc = x_loc.clone()
    x_s = x_s.clone()
    lam = torch.full((1,), float(lam0), dtype=torch.float64, device=dev)
    costs = torch.empty(max(int(n_iter), 0), dtype=torch.float64, device=dev)
    c = red(steps.normal(x_loc, x_s).clone())

    def iteration(last):
        sums = red(steps.eliminate(lam))
        d_loc, d_s = steps.back(sums, lam)
        xt = torch.minimum(torch.maximum(x_loc + d_loc, lo_l), hi_l)
        xst = torch.minimum(torch.maximum(x_s + d_s, lo_s), hi_s)
        ct = red(steps.costs(xt, xst).sum().reshape(1))
        better = ct < c
        x_loc.copy_(torch.where(better, xt, x_loc))
        x_s.copy_(torch.where(better, xst, x_s))
        lam.copy_(torch.where(better, lam * 0.5, lam * 3.0))
        if last:
            c.copy_(torch.where(better, ct, c))
        else:
            c.copy_(torch.where(better, red(steps.normal(x_loc, x_s, better).clone()), c))

    n_iter = int(n_iter)
    it = 0
    if graph and allsum is None and callback is None and n_iter >= 3 and dev.type == "cuda":
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            iteration(False)                          # the first iteration eagerly (warms every buffer up)
            costs[0].copy_(c[0])
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                iteration(False)
        torch.cuda.current_stream().wait_stream(side)
        for it in range(1, n_iter - 1):
            g.replay()
            costs[it].copy_(c[0])
        del g
        it = n_iter - 1
    while it < n_iter:
        iteration(it + 1 == n_iter)
        costs[it].copy_(c[0])
        if callback is not None:
            callback(it, float(c[0].item()))
        it += 1
    return x_loc, x_s, costs


def fit_joint_uneven(batch: UnevenBatch, spec, z_meas: Sequence[np.ndarray], n_iter: int = 30,
                     x0_phys: Optional[np.ndarray] = None, x0_shared: Optional[float] = None, lam0: float = 1e-2,
                     callback: Optional[Callable[[int, float], None]] = None, group=None,
                     graph: bool = True) -> UnevenFitResult:
    """Joint LM over an uneven batch: every `scope="sample"` slot free per voxel (where its field and pool
    exist), at most one `scope="shared"` slot common to all voxels; plain values only. z_meas[i] holds
    voxel i's measured Z (its table's rows). One damping for the whole problem, accept if the summed
    squared residual falls (lam x 0.5) else lam x 3 (fitting/joint.py:149-162, 359-453).

    Every iteration runs on the device with no value read back (`_joint_lm`); with `graph` (one GPU, no
    callback) one iteration is captured in a CUDA graph and replayed.

    `group`: a torch.distributed process group whose ranks each hold their own voxels (one GPU per
    rank). The shared value is then common to the voxels of every rank: each iteration all-reduces four
    numbers (the Schur sums of the shared column) and the costs, so every rank takes the same steps."""
    torch = _lib.torch_cuda()
    loc = [l for l, s in enumerate(spec.slots) if s.scope == "sample"]
    shr = [l for l, s in enumerate(spec.slots) if s.scope == "shared"]
    bad = [s.name for s in spec.slots if s.scope not in ("sample", "shared") or s.mode != "value" or s.samples]
    if bad or len(shr) > 1 or not loc:
        raise ValueError(f"fit_joint_uneven: sample-scope plain values plus at most one shared value; got {bad or shr}")
    if len(loc) > 8:
        raise ValueError(f"fit_joint_uneven: at most 8 values per voxel, got {len(loc)}")
    n, PL, S = batch.n, len(loc), len(shr)
    if len(z_meas) != n:
        raise ValueError(f"z_meas has {len(z_meas)} voxels, the batch {n}")
    steps = _JointSteps(batch, spec, z_meas, loc, shr)
    scl = spec.scales
    lo, hi = spec.lo_phys / scl, spec.hi_phys / scl
    x0 = np.broadcast_to(spec.x0_phys[loc] if x0_phys is None else np.asarray(x0_phys, np.float64), (n, PL))
    f64 = dict(dtype=torch.float64, device="cuda")
    x_loc = torch.as_tensor(np.ascontiguousarray(x0 / scl[loc])).cuda()
    xs0 = float((spec.x0_phys[shr[0]] if x0_shared is None else x0_shared) / scl[shr[0]]) if S else 0.0
    x_s = torch.tensor([xs0], **f64)
    lo_l, hi_l = torch.as_tensor(lo[loc]).cuda(), torch.as_tensor(hi[loc]).cuda()
    lo_s = torch.tensor([lo[shr[0]] if S else 0.0], **f64)
    hi_s = torch.tensor([hi[shr[0]] if S else 0.0], **f64)
    allsum = None
    if group is not None:
        import torch.distributed as dist

        def allsum(t):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
            return t
    x_loc, x_s, costs = _joint_lm(steps, x_loc, x_s, lo_l, hi_l, lo_s, hi_s, lam0, n_iter, allsum,
                                  graph=graph and group is None, callback=callback)
    per = steps.costs(x_loc, x_s).cpu().numpy()
    npts = np.zeros(n)
    for g in batch.groups:
        npts[g.voxels] = np.diff(g.chain_start)
    X = x_loc.cpu().numpy() * scl[loc]
    X[steps.free_np == 0] = np.nan
    xs = float(x_s.cpu().numpy()[0])
    return UnevenFitResult(X, (xs * scl[shr[0]]) if S else None, np.sqrt(per / npts), costs.cpu().numpy(),
                           [spec.slots[l].name for l in loc], spec.slots[shr[0]].name if S else None)
