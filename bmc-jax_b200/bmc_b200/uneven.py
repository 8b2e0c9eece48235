"""Uneven batches: voxels with their own pool counts and event tables, simulated and fitted together.

BMC-JAX runs one event table per Experiment (fitting/experiment.py:43-46) and one pool count per
parameter batch, so a mix of models and protocols is one call per shape class there. Here the voxels of
a pool count share one launch whatever their tables (bmc_uneven_* in include/bmc_b200.h); each voxel
gets the result its own class's call gives. `fit_joint_uneven` fits per-voxel values plus at most one
value shared by every voxel (e.g. water T1) with the joint Levenberg-Marquardt of fitting/joint.py:
149-162 -- one damping for the whole problem, the same damped normal equations -- assembled per voxel
on the GPU and solved through the Schur complement of the shared column (bmc_normal_segments,
bmc_schur_step). The loop runs on the host with every array on the device; one number (the cost)
comes back per iteration.
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

    def run(self, params, m0, tangents=None, jz=None, spread=None):
        """z [n_chains] (device) for params [n_fields][n_voxels] and m0 [n_voxels][N] (device, float64);
        with tangents, their derivatives into jz [n_tangents][n_chains]; `spread` a _lib.Spread or None."""
        torch = _lib.torch_cuda()
        z = torch.empty(self.n_chains, dtype=torch.float64, device="cuda")
        _lib.check(_lib.lib().bmc_uneven_simulate(self.plan, _lib.ptr(params), _lib.ptr(m0),
                                                  None if spread is None else C.byref(spread),
                                                  None if tangents is None else C.byref(tangents), _lib.ptr(z),
                                                  _lib.ptr(jz), _lib.stream_handle()))
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
        for e in exps:
            k = _table_key(e.events)
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


def fit_joint_uneven(batch: UnevenBatch, spec, z_meas: Sequence[np.ndarray], n_iter: int = 30,
                     x0_phys: Optional[np.ndarray] = None, x0_shared: Optional[float] = None, lam0: float = 1e-2,
                     callback: Optional[Callable[[int, float], None]] = None, group=None) -> UnevenFitResult:
    """Joint LM over an uneven batch: every `scope="sample"` slot free per voxel (where its field and pool
    exist), at most one `scope="shared"` slot common to all voxels; plain values only. z_meas[i] holds
    voxel i's measured Z (its table's rows). One damping for the whole problem, accept if the summed
    squared residual falls (lam x 0.5) else lam x 3 (fitting/joint.py:149-162, 359-453).

    `group`: a torch.distributed process group whose ranks each hold their own voxels (one GPU per
    rank). The shared value is then common to the voxels of every rank: each iteration all-reduces four
    numbers (the Schur sums of the shared column) and the costs, so every rank takes the same steps."""
    from .fitting import field_row
    torch = _lib.torch_cuda()
    loc = [l for l, s in enumerate(spec.slots) if s.scope == "sample"]
    shr = [l for l, s in enumerate(spec.slots) if s.scope == "shared"]
    bad = [s.name for s in spec.slots if s.scope not in ("sample", "shared") or s.mode != "value" or s.samples]
    if bad or len(shr) > 1 or not loc:
        raise ValueError(f"fit_joint_uneven: sample-scope plain values plus at most one shared value; got {bad or shr}")
    if len(loc) > 8:
        raise ValueError(f"fit_joint_uneven: at most 8 values per voxel, got {len(loc)}")
    n, PL, S = batch.n, len(loc), len(shr)
    P = PL + S
    if len(z_meas) != n:
        raise ValueError(f"z_meas has {len(z_meas)} voxels, the batch {n}")
    scl = spec.scales
    lo, hi = spec.lo_phys / scl, spec.hi_phys / scl
    x0 = np.broadcast_to(spec.x0_phys[loc] if x0_phys is None else np.asarray(x0_phys, np.float64), (n, PL))
    x_loc = torch.as_tensor(x0 / scl[loc]).cuda()
    x_s = float((spec.x0_phys[shr[0]] if x0_shared is None else x0_shared) / scl[shr[0]]) if S else 0.0
    lo_l, hi_l = torch.as_tensor(lo[loc]).cuda(), torch.as_tensor(hi[loc]).cuda()
    free = np.zeros((n, PL))
    for g in batch.groups:
        g.rows = []
        for j, l in enumerate(loc):
            s = spec.slots[l]
            ok = s.index is None or s.index < g.nc
            g.rows.append(field_row(s.field, s.index, g.nc) if ok else None)
            if ok:
                free[g.voxels, j] = 1.0
        g.row_s = field_row(spec.slots[shr[0]].field, spec.slots[shr[0]].index, g.nc) if S else None
        for k, v in enumerate(g.voxels):
            zv = np.asarray(z_meas[v], np.float64).reshape(-1)
            if zv.size != g.chain_start[k + 1] - g.chain_start[k]:
                raise ValueError(f"z_meas[{v}] has {zv.size} points, its table {g.chain_start[k + 1] - g.chain_start[k]}")
        g.zm = torch.as_tensor(np.concatenate([np.asarray(z_meas[v], np.float64).reshape(-1) for v in g.voxels])).cuda()
        g.idx = torch.as_tensor(g.voxels).cuda()
        g.seg = torch.repeat_interleave(torch.arange(len(g.voxels), device="cuda"),
                                        torch.as_tensor(np.diff(g.chain_start)).cuda())
        # tangents: the local slots (zero where a slot does not apply) then the shared one
        tg = _lib.Tangents()
        tg.n_tangents = P
        seed = np.zeros((P, len(g.voxels)))
        for j, l in enumerate(loc):
            tg.field_row[j] = _lib.SEED_NONE if g.rows[j] is None else g.rows[j]
            if g.rows[j] is not None:
                seed[j] = scl[l]
        if S:
            tg.field_row[PL] = g.row_s
            seed[PL] = scl[shr[0]]
        g.seed = torch.as_tensor(seed).cuda()
        tg.d_seed = g.seed.data_ptr()
        tg.d_dm0 = None
        g.tangents = tg
        g.jz = torch.empty((P, g.n_chains), dtype=torch.float64, device="cuda")
    d_free = torch.as_tensor(free).cuda()

    def params_at(g, xl, xs):
        p = g.params.clone()
        xv = xl.index_select(0, g.idx)
        for j, l in enumerate(loc):
            if g.rows[j] is not None:
                p[g.rows[j]] = xv[:, j] * scl[l]
        if S:
            p[g.row_s] = xs * scl[shr[0]]
        return p

    H = torch.empty((n, P, P), dtype=torch.float64, device="cuda")
    gr = torch.empty((n, P), dtype=torch.float64, device="cuda")
    cv = torch.empty(n, dtype=torch.float64, device="cuda")
    work = torch.empty((2 * PL + 4) * n + 4, dtype=torch.float64, device="cuda")
    sums = torch.empty(4, dtype=torch.float64, device="cuda")
    if group is not None:
        import torch.distributed as dist
        allsum = lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    else:
        allsum = None

    def total(v: float) -> float:
        if allsum is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        allsum(t)
        return float(t.item())
    d_loc = torch.empty((n, PL), dtype=torch.float64, device="cuda")
    d_s = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = _lib.lib()

    def normal(xl, xs):
        for g in batch.groups:
            z = g.run(params_at(g, xl, xs), g.tangents, g.jz)
            r = z - g.zm
            Hg = torch.empty((len(g.voxels), P, P), dtype=torch.float64, device="cuda")
            gg = torch.empty((len(g.voxels), P), dtype=torch.float64, device="cuda")
            cg = torch.empty(len(g.voxels), dtype=torch.float64, device="cuda")
            _lib.check(L.bmc_normal_segments(len(g.voxels), P, g.n_chains, _lib.ptr(g.d_chain_start), _lib.ptr(g.jz),
                                             _lib.ptr(r), _lib.ptr(Hg), _lib.ptr(gg), _lib.ptr(cg),
                                             _lib.stream_handle()))
            H[g.idx], gr[g.idx], cv[g.idx] = Hg, gg, cg
        return total(float(cv.sum().item()))

    def cost_at(xl, xs, per_voxel=False):
        out = torch.empty(n, dtype=torch.float64, device="cuda")
        for g in batch.groups:
            r = g.run(params_at(g, xl, xs)) - g.zm
            out[g.idx] = torch.zeros(len(g.voxels), dtype=torch.float64, device="cuda").index_add_(0, g.seg, r * r)
        return out if per_voxel else total(float(out.sum().item()))

    lam = float(lam0)
    costs = []
    c = normal(x_loc, x_s)
    for it in range(int(n_iter)):
        if allsum is None:
            _lib.check(L.bmc_schur_step(n, PL, S, _lib.ptr(H), _lib.ptr(gr), _lib.ptr(d_free), lam, _lib.ptr(d_loc),
                                        _lib.ptr(d_s), _lib.ptr(work), _lib.stream_handle()))
        else:
            _lib.check(L.bmc_schur_eliminate(n, PL, S, _lib.ptr(H), _lib.ptr(gr), _lib.ptr(d_free), lam,
                                             _lib.ptr(work), _lib.ptr(sums), _lib.stream_handle()))
            allsum(sums)
            _lib.check(L.bmc_schur_back(n, PL, S, _lib.ptr(sums), lam, _lib.ptr(work), _lib.ptr(d_loc), _lib.ptr(d_s),
                                        _lib.stream_handle()))
        xt = torch.minimum(torch.maximum(x_loc + d_loc, lo_l), hi_l)
        xst = float(np.clip(x_s + float(d_s.item()), lo[shr[0]], hi[shr[0]])) if S else 0.0
        ct = cost_at(xt, xst)
        if ct < c:
            x_loc, x_s, lam = xt, xst, lam * 0.5
            c = normal(x_loc, x_s) if it + 1 < n_iter else ct
        else:
            lam = lam * 3.0
        costs.append(c)
        if callback is not None:
            callback(it, c)
    per = cost_at(x_loc, x_s, per_voxel=True).cpu().numpy()
    npts = np.zeros(n)
    for g in batch.groups:
        npts[g.voxels] = np.diff(g.chain_start)
    X = x_loc.cpu().numpy() * scl[loc]
    X[free == 0] = np.nan
    return UnevenFitResult(X, (x_s * scl[shr[0]]) if S else None, np.sqrt(per / npts), np.asarray(costs),
                           [spec.slots[l].name for l in loc], spec.slots[shr[0]].name if S else None)
