"""Fitting: BMC-JAX's `bmc_jax.fitting` API on the B200 kernels.

  FreeParam, FitSpec, write_params   which parameters are free    (fitting/params.py:38-112)
  Experiment                         what is simulated            (fitting/experiment.py:21-141)
  levenberg_marquardt                bounded LM, physics-free     (fitting/lm.py:20-67)
  fit, fit_batch                     every sample alone           (fitting/independent.py:51-129, 226-298)
  fit_joint                          shared / per-block / partly free values (fitting/joint.py:165-453)
  FitResult                          what comes back              (fitting/result.py:23-174)

`fit` and `fit_batch` run every LM iteration of every voxel on the GPU (bmc_lm_fit): residual,
forward-mode Jacobian, float64 normal equations, damped solve, clip, trial residual, accept/reject.
`fit_joint` without a shared or per-block value is the same device loop with per-sample holds; with
one, the samples are coupled and one damping governs the joint step: the host loop of the reference
(joint.py:375-416) with per-sample Jacobians from the GPU and the joint normal equations solved by a
Schur complement over the shared columns (the same linear system as the reference's dense solve).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .simulation import (SimParams, SimEvent, EventType, pad_events, tile_params, n_cest_of, n_samples,
                         pack_params, state_size, DeviceEvents, problem, initial_state, B0Spread, _device)

__all__ = ["Experiment", "FreeParam", "FitSpec", "write_params", "levenberg_marquardt", "fit", "fit_batch",
           "fit_joint", "FitResult"]

PSEUDO = ("m_start", "b0_spread")
_SCALAR_FIELDS = ("water_r1", "water_r2", "water_f", "mt_k", "mt_f", "mt_dw", "mt_r1", "mt_r2", "mt_lineshape",
                  "b0", "gamma", "b0_inhom", "rel_b1")
_POOL_FIELDS = ("cest_k", "cest_f", "cest_dw", "cest_r1", "cest_r2")


def field_row(field: str, index: Optional[int], n_cest: int) -> int:
    """Row of a SimParams field value in the C ABI's params layout."""
    if field in _POOL_FIELDS:
        if index is None or not 0 <= int(index) < n_cest:
            raise ValueError(f"{field}: pool index {index} outside 0..{n_cest - 1}")
        return 3 + _POOL_FIELDS.index(field) * n_cest + int(index)
    if field in ("water_r1", "water_r2", "water_f"):
        return ("water_r1", "water_r2", "water_f").index(field)
    if field in _SCALAR_FIELDS:
        return 3 + 5 * n_cest + _SCALAR_FIELDS[3:].index(field)
    raise ValueError(f"{field}: not a SimParams field")


# ------------------------------------------------------------------------------------------------
# which parameters are free (fitting/params.py)
# ------------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class FreeParam:
    name: str
    field: str
    index: Optional[int]
    scale: float
    lo: float
    hi: float
    x0: float
    scope: str = "sample"
    samples: Optional[Tuple[int, ...]] = None
    mode: str = "value"

    def __post_init__(self):
        if self.scope not in ("sample", "shared", "block"):
            raise ValueError(f"{self.name}: scope {self.scope!r}; use 'sample', 'shared' or 'block'")
        if self.mode not in ("value", "factor", "add"):
            raise ValueError(f"{self.name}: mode {self.mode!r}; use 'value', 'factor' or 'add'")
        if self.field == "m_start" and (self.index is not None or self.mode == "add"):
            raise ValueError(f"{self.name}: m_start is one number per sample (index None), as a value or a factor")
        if self.field == "b0_spread" and (self.index is not None or self.mode != "value"):
            raise ValueError(f"{self.name}: b0_spread is one width in Hz (index None, mode 'value')")
        if self.samples is not None:
            object.__setattr__(self, "samples", tuple(sorted({int(i) for i in self.samples})))
            if not self.samples:
                raise ValueError(f"{self.name}: samples=() frees it nowhere; leave it out of the spec")


@dataclass(frozen=True)
class FitSpec:
    slots: List[FreeParam]

    @property
    def n(self):
        return len(self.slots)

    @property
    def scales(self):
        return np.array([s.scale for s in self.slots], np.float64)

    @property
    def lo_phys(self):
        return np.array([s.lo for s in self.slots], np.float64)

    @property
    def hi_phys(self):
        return np.array([s.hi for s in self.slots], np.float64)

    @property
    def x0_phys(self):
        return np.array([s.x0 for s in self.slots], np.float64)

    def to_scaled(self, x_phys):
        return np.asarray(x_phys) / self.scales

    def to_phys(self, x_scaled):
        return np.asarray(x_scaled) * self.scales

    @property
    def independent(self) -> bool:
        return all(s.scope == "sample" and s.samples is None and s.mode == "value" and s.field not in PSEUDO
                   for s in self.slots)

    def require_independent(self, caller: str) -> None:
        if not self.independent:
            joint = [s.name for s in self.slots if s.scope != "sample" or s.samples is not None
                     or s.mode != "value" or s.field in PSEUDO]
            raise ValueError(f"{caller}: {joint} are shared, per block, free in some samples only, a factor / an "
                             "offset, m_start or b0_spread (FreeParam scope / samples / mode / field), which "
                             "samples fitted alone with plain values cannot do; use fit_joint")


def write_params(base: SimParams, x_scaled, spec: FitSpec) -> SimParams:
    """Scaled x -> physical values written into the named fields (fitting/params.py:100-112)."""
    x_phys = np.asarray(x_scaled, np.float64) * spec.scales
    upd = {}
    for i, s in enumerate(spec.slots):
        if s.index is None:
            upd[s.field] = x_phys[..., i]
        else:
            cur = np.array(upd.get(s.field, getattr(base, s.field)), np.float64, copy=True)
            cur[..., s.index] = x_phys[..., i]
            upd[s.field] = cur
    return base._replace(**upd)


# ------------------------------------------------------------------------------------------------
# what is simulated (fitting/experiment.py)
# ------------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class Experiment:
    """Parameters, a sequence, a starting state, and the index of water's Mz."""
    params: object
    events: SimEvent
    m0: object
    mz_loc: int

    @property
    def n_offsets(self) -> int:
        return int(np.shape(self.events.dt)[0])

    @property
    def n_events(self) -> int:
        return int(np.shape(self.events.dt)[1])

    def simulate(self) -> np.ndarray:
        """Water Mz at every offset: (n_offsets,) for one sample, (n_samples, n_offsets) for a batch."""
        from .simulation import simulate_z
        return simulate_z(self.params, self.events, self.m0, self.mz_loc)

    @classmethod
    def from_parameters(cls, params, events) -> "Experiment":
        from .simulation import to_sim_params
        jp = to_sim_params(params)
        scale = float(getattr(params.options, "scale", 1.0))
        return cls(jp, events, initial_state(jp, scale), params.mz_loc)

    @classmethod
    def stack(cls, experiments: Sequence["Experiment"]) -> "Experiment":
        experiments = list(experiments)
        if not experiments:
            raise ValueError("stack needs at least one experiment")
        locs = {p.mz_loc for p in experiments}
        if len(locs) > 1:
            raise ValueError(f"experiments disagree on mz_loc: {sorted(locs)}; they must describe "
                             "the same pools in the same order")
        width = max(p.n_events for p in experiments)
        padded = [pad_events(p.events, width) for p in experiments]
        events = SimEvent(*[np.concatenate([np.asarray(getattr(e, f)) for e in padded], axis=0)
                            for f in SimEvent._fields])
        first = experiments[0]
        return cls(first.params, events, first.m0, first.mz_loc)


# ------------------------------------------------------------------------------------------------
# what comes back (fitting/result.py)
# ------------------------------------------------------------------------------------------------
def _near(x, ref, rel, floor):
    """|x - ref| <= floor + rel |ref|, elementwise (NaN compares False)."""
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    return np.abs(x - ref) <= floor + rel * np.abs(ref)


def _rms_rows(r):
    """Root mean square over the last axis."""
    r = np.asarray(r, np.float64)
    return np.linalg.norm(r, axis=-1) / np.sqrt(max(r.shape[-1], 1))


@dataclass(frozen=True)
class FitResult:
    """The outcome of `fit` / `fit_joint` (the fields of BMC-JAX fitting/result.py:23-174).

    x (n_samples, n_params) fitted values in physical units; z_fit the model at x and z_meas the data it
    was fitted to; spec the FitSpec (names, bounds). n_per_block: offsets per stacked experiment (for
    rms_per_block). fit_joint also fills free (where a slot was fitted; elsewhere x holds the value the
    sample carries), sd and corr (misfit-scaled standard deviations and correlations, NaN where not
    free), x0, cost (after every step), nan_steps and blocks (per-experiment values, name -> dict of x,
    sd and at_bounds; their column of x is NaN)."""
    x: np.ndarray
    z_fit: np.ndarray
    z_meas: np.ndarray
    spec: FitSpec
    n_per_block: Optional[int] = None
    free: Optional[np.ndarray] = None
    sd: Optional[np.ndarray] = None
    corr: Optional[np.ndarray] = None
    x0: Optional[np.ndarray] = None
    cost: Optional[np.ndarray] = None
    nan_steps: int = 0
    blocks: Optional[dict] = None

    @property
    def names(self) -> List[str]:
        return [slot.name for slot in self.spec.slots]

    def __getitem__(self, name: str) -> np.ndarray:
        """One parameter over the samples (a per-block parameter: over the experiments)."""
        if name in (self.blocks or {}):
            return self.blocks[name]["x"]
        col = {nm: j for j, nm in enumerate(self.names)}.get(name)
        if col is None:
            raise KeyError(f"no parameter {name!r}; the fit has {self.names}")
        return self.x[:, col]

    @property
    def residual(self) -> np.ndarray:
        """z_fit - z_meas."""
        return np.asarray(self.z_fit) - np.asarray(self.z_meas)

    @property
    def rms(self) -> np.ndarray:
        return _rms_rows(self.residual)

    @property
    def rms_per_block(self):
        """(n_samples, n_blocks) rms of every stacked experiment, or None without n_per_block."""
        if self.n_per_block is None:
            return None
        m = int(self.n_per_block)
        r = self.residual
        nb = r.shape[-1] // m
        return np.stack([_rms_rows(r[..., b * m:(b + 1) * m]) for b in range(nb)], axis=-1)

    def _only_free(self, mask):
        return mask if self.free is None else mask & np.asarray(self.free, bool)

    @property
    def at_bounds(self) -> np.ndarray:
        """Fitted values that sit on a bound (within 1e-8 + 1e-5 of it): not measurements."""
        lo = np.asarray(self.spec.lo_phys)[None, :]
        hi = np.asarray(self.spec.hi_phys)[None, :]
        return self._only_free(_near(self.x, lo, 1e-5, 1e-8) | _near(self.x, hi, 1e-5, 1e-8))

    @property
    def unmoved(self):
        """Free values that never left their start (within 1e-6 relative), or None without x0."""
        if self.x0 is None:
            return None
        return self._only_free(_near(self.x, self.x0, 1e-6, 0.0))

    def summary(self) -> str:
        """A text table: one line per sample, a flag after every value that is railed ([b]) or held
        ([h]), then the per-experiment values."""
        names = self.names
        w = max([10] + [len(n) + 4 for n in names])
        railed, held = self.at_bounds, (None if self.free is None else ~np.asarray(self.free, bool))
        lines = [f"FitResult: {self.x.shape[0]} samples, mean rms {float(np.mean(self.rms)):.3e}",
                 "sample | " + " ".join(n.rjust(w) for n in names) + " |       rms"]
        for i, row in enumerate(np.asarray(self.x)):
            cells = []
            for j, v in enumerate(row):
                tag = "[b]" if railed[i, j] else ("[h]" if held is not None and held[i, j] else "   ")
                cells.append(f"{v:.5g}{tag}".rjust(w))
            lines.append(f"{i:6d} | " + " ".join(cells) + f" | {self.rms[i]:9.2e}")
        if railed.any() or (held is not None and held.any()):
            lines.append("[b] on a bound: the optimiser was stopped there, not a measurement; "
                         "[h] held: not free in this sample")
        for name, blk in (self.blocks or {}).items():
            vals = ", ".join(f"{v:.5g}" + (" [b]" if r else "") for v, r in zip(blk["x"], blk["at_bounds"]))
            lines.append(f"{name} per experiment: {vals}")
        return "\n".join(lines)

    def __repr__(self) -> str:
        n_rail = int(np.count_nonzero(self.at_bounds))
        tail = f", {n_rail} values on a bound" if n_rail else ""
        return (f"<FitResult of {self.x.shape[0]} samples: {', '.join(self.names)}; "
                f"mean rms {float(np.mean(self.rms)):.3e}{tail}>")


# ------------------------------------------------------------------------------------------------
# bounded LM without physics (fitting/lm.py:20-67), for any residual function on the host
# ------------------------------------------------------------------------------------------------
def levenberg_marquardt(resid_fn, x0, lo, hi, n_iter=40, lam0=1e-2, use_fwd=False, return_trajectory=False,
                        free=None, jac_fn=None):
    """Damped Gauss-Newton for one residual vector, fixed iterations with accept/reject, float64.

    The step rule is the reference's exactly. `jac_fn(x)` gives the Jacobian; without it a central
    difference is used (this entry point is physics-free: the BMC fits use the GPU's exact tangents)."""
    x = np.asarray(x0, np.float64).copy()
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    P = x.size
    fr = None if free is None else np.asarray(free, np.float64)

    def jac(x):
        if jac_fn is not None:
            return np.asarray(jac_fn(x), np.float64)
        r0 = np.asarray(resid_fn(x), np.float64)
        J = np.empty((r0.size, P))
        for j in range(P):
            h = 1e-7 * max(1.0, abs(x[j]))
            e = np.zeros(P)
            e[j] = h
            J[:, j] = (np.asarray(resid_fn(x + e)) - np.asarray(resid_fn(x - e))) / (2 * h)
        return J

    lam = float(lam0)
    X, Cs = [], []
    for _ in range(n_iter):
        r = np.asarray(resid_fn(x), np.float64)
        c = float(r @ r)
        J = jac(x)
        if fr is not None:
            J = J * fr
        g, H = J.T @ r, J.T @ J
        A = H + lam * (np.diag(np.diag(H)) + 1e-9 * np.eye(P))
        if fr is not None:
            A = A + np.diag(1.0 - fr)
        xn = np.clip(x + np.linalg.solve(A, -g), lo, hi)
        rn = np.asarray(resid_fn(xn), np.float64)
        cn = float(rn @ rn)
        better = cn < c
        x = xn if better else x
        lam = lam * 0.5 if better else lam * 3.0
        X.append(x.copy())
        Cs.append(cn if better else c)
    if return_trajectory:
        return x, np.array(X), np.array(Cs)
    return x


# ------------------------------------------------------------------------------------------------
# the device LM (bmc_lm_fit)
# ------------------------------------------------------------------------------------------------
def _lm_device(params_b: SimParams, events: SimEvent, m0_b, mz: int, rows, modes, scales, lo, hi, z_meas, X0,
               n_iter: int, lam0: float, skip: int = 0, free=None, spread=None, sigma=None):
    """Run bmc_lm_fit; returns (x scaled (n, P), cost trajectory (n, n_iter))."""
    torch = _lib.torch_cuda()
    n = n_samples(params_b)
    nc = n_cest_of(params_b)
    N = state_size(nc)
    P = len(rows)
    if P > _lib.MAX_TANGENTS:
        raise ValueError(f"at most {_lib.MAX_TANGENTS} free parameters per sample, got {P}")
    dev_ev = DeviceEvents(events)
    pdev = _device(pack_params(params_b, n))
    mdev = _device(np.broadcast_to(np.asarray(m0_b, np.float64), (n, N)))
    zdev = _device(z_meas)
    xdev = _device(X0)
    fdev = None if free is None else _device(np.asarray(free, np.float64))
    xout = torch.empty((n, P), dtype=torch.float64, device="cuda")
    ctraj = torch.empty((n, max(n_iter, 1)), dtype=torch.float64, device="cuda")
    spec = _lib.FitSpecC()
    spec.n_params, spec.n_iter, spec.lam0 = P, int(n_iter), float(lam0)
    for p in range(P):
        spec.field_row[p], spec.mode[p] = int(rows[p]), int(modes[p])
        spec.scale[p], spec.lo[p], spec.hi[p] = float(scales[p]), float(lo[p]), float(hi[p])
    spec.d_free = None if fdev is None else fdev.data_ptr()
    spec.n_points_skip = int(skip)
    sp, keep = (None, None)
    if spread is not None:
        u, w = spread.nodes_weights()
        sdev = _device(np.broadcast_to(np.asarray(sigma, np.float64), (n,)))
        sp, keep = _lib.spread_struct(u, w, sdev)
    pr = problem(n, dev_ev.n_offsets, dev_ev.n_events, nc, int(mz), _lib.F64)
    _lib.check(_lib.lib().bmc_lm_fit(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev), sp, spec, _lib.ptr(zdev),
                                     _lib.ptr(xdev), _lib.ptr(xout), _lib.ptr(ctraj), None, _lib.stream_handle()))
    x = xout.cpu().numpy()
    c = ctraj.cpu().numpy()[:, :n_iter]
    del keep
    return x, c


def _slot_rows(spec: FitSpec, nc: int):
    rows, modes = [], []
    for s in spec.slots:
        if s.field == "m_start":
            rows.append(_lib.SLOT_M_START)
        elif s.field == "b0_spread":
            rows.append(_lib.SLOT_SPREAD_SIGMA)
        else:
            rows.append(field_row(s.field, s.index, nc))
        modes.append({"value": 0, "factor": 1, "add": 2}[s.mode])
    return rows, modes


def _batched(params, n):
    return params if n_samples(params) is not None else tile_params(params, n)


def fit_batch(base, events, M0_batch, water_z, spec: FitSpec, z_meas_batch, X0_phys=None, n_iter=40,
              skip_first=True, base_batched=False, use_fwd=None, max_chunk=None, dtype=None):
    """Every voxel with damped Gauss-Newton, all on the GPU (independent.py:51-129). Returns physical
    X (n, P). The Jacobian is always forward mode (use_fwd is accepted for compatibility); `dtype`
    is accepted and ignored: fits run in float64."""
    spec.require_independent("fit_batch")
    z = np.asarray(z_meas_batch, np.float64)
    n_vox = z.shape[0]
    base_b = base if base_batched else tile_params(base, n_vox)
    nc = n_cest_of(base_b)
    N = state_size(nc)
    M0_b = np.asarray(M0_batch, np.float64)
    if M0_b.ndim == 1:
        M0_b = np.broadcast_to(M0_b, (n_vox,) + M0_b.shape)
    if M0_b.shape[0] != n_vox:
        raise ValueError(f"M0_batch has {M0_b.shape[0]} rows for {n_vox} voxels")
    skip = 1 if skip_first else 0
    z_t = z[:, skip:]
    scales = spec.scales
    lo, hi = spec.lo_phys / scales, spec.hi_phys / scales
    X0 = (np.broadcast_to(spec.to_scaled(spec.x0_phys), (n_vox, spec.n)) if X0_phys is None
          else np.broadcast_to(spec.to_scaled(X0_phys), (n_vox, spec.n)))
    rows, modes = _slot_rows(spec, nc)
    chunk = max_chunk or n_vox
    parts = []
    for a in range(0, n_vox, chunk):
        b = min(a + chunk, n_vox)
        sub = SimParams(*[np.asarray(v)[a:b] for v in base_b])
        x, _ = _lm_device(sub, events, M0_b[a:b], water_z, rows, modes, scales, lo, hi, z_t[a:b], X0[a:b],
                          n_iter, 1e-2, skip)
        parts.append(x)
    return np.concatenate(parts) * scales


def fit(experiment: Experiment, spec: FitSpec, z_meas, n_iter=30, x0_phys=None, n_per_block=None, **kwargs):
    """Fit `spec`'s parameters of `experiment` to `z_meas` (independent.py:226-298)."""
    from .simulation import simulate_z
    spec.require_independent("fit")
    z = np.atleast_2d(np.asarray(z_meas, np.float64))
    n = z.shape[0]
    base = _batched(experiment.params, n)
    m0 = np.asarray(experiment.m0, np.float64)
    if m0.ndim == 1:
        m0 = np.broadcast_to(m0, (n,) + m0.shape)
    X = fit_batch(base, experiment.events, m0, experiment.mz_loc, spec, z, X0_phys=x0_phys, n_iter=n_iter,
                  skip_first=False, base_batched=True, **kwargs)
    z_fit = simulate_z(write_params(base, spec.to_scaled(X), spec), experiment.events, m0, experiment.mz_loc,
                       precision=_lib.F64)
    return FitResult(X, np.asarray(z_fit), z, spec, n_per_block)


# ------------------------------------------------------------------------------------------------
# joint fits (fitting/joint.py)
# ------------------------------------------------------------------------------------------------
@dataclass
class _Columns:
    """Where every free number of a joint fit lives.

    Sample i's local vector has one entry per slot, or one per experiment for a per-block slot, the slot's
    entries starting at pos[slot]. A joint column is one free number: a sample value (one sample), a
    shared value (every sample it is free in) or one experiment's value of a per-block slot; `cols` lists
    (slot, samples, experiment or -1) per column and col_of[i, j] names the column behind sample i's local
    entry j (-1: held)."""
    free: np.ndarray
    pos: np.ndarray
    n_loc: int
    cols: list
    col_of: np.ndarray


def _columns(spec: FitSpec, n: int, n_blocks: int) -> _Columns:
    widths = [n_blocks if sl.scope == "block" else 1 for sl in spec.slots]
    pos = np.cumsum([0] + widths[:-1]).astype(int)
    n_loc = int(sum(widths))
    free = np.zeros((n, spec.n), bool)
    col_of = np.full((n, n_loc), -1, int)
    cols = []
    for l, sl in enumerate(spec.slots):
        who = np.arange(n) if sl.samples is None else np.asarray(sl.samples, int)
        outside = who[(who < 0) | (who >= n)]
        if outside.size:
            raise ValueError(f"{sl.name}: samples {outside.tolist()} do not exist (the fit has {n})")
        free[who, l] = True
        if sl.scope == "sample":                 # one column per sample
            for i in who.tolist():
                col_of[i, pos[l]] = len(cols)
                cols.append((l, [i], -1))
        else:                                    # one column for all its samples, per experiment if "block"
            for b in (range(n_blocks) if sl.scope == "block" else (-1,)):
                col_of[who, pos[l] + max(b, 0)] = len(cols)
                cols.append((l, who.tolist(), b))
    return _Columns(free, pos, n_loc, cols, col_of)


def _carried(params: SimParams, m0, spec: FitSpec, sig_held):
    """(n, L): the number each slot stands for where it is not free -- the field's own value, 1 for a
    factor, 0 for an offset, the start state's water Mz over water_f for m_start, the held width for
    b0_spread (fitting/joint.py:99-117)."""
    n = m0.shape[0]
    water_z = 2 * (1 + n_cest_of(params))
    neutral = {"factor": 1.0, "add": 0.0}

    def held(sl):
        if sl.field == "b0_spread":
            return np.broadcast_to(np.asarray(sig_held, np.float64), (n,))
        if sl.mode in neutral:
            return np.full(n, neutral[sl.mode])
        if sl.field == "m_start":
            return m0[:, water_z] / np.asarray(params.water_f, np.float64)
        v = np.asarray(getattr(params, sl.field), np.float64)
        return v if sl.index is None else v[:, sl.index]
    return np.column_stack([held(sl) for sl in spec.slots])


def _error_bars(Hl, resid, lay: _Columns, spec: FitSpec, coupled: bool, x_cols=None):
    """Misfit-scaled standard deviations and correlations at the solution (fitting/joint.py:418-453), from
    each sample's local normal matrix Hl[i] = J_i^T J_i: (sd (n, L), corr (n, L, L), per-block dict).

    Independent samples: cov_i = pinv(H_i over its free slots) s_i^2 with s_i^2 = r_i.r_i / (points - free).
    Coupled: J^T J over the joint columns is the sum of the samples' blocks placed at their columns, and
    cov = pinv(J^T J) s^2 with s^2 = r.r / (all points - columns); a sample's slots read their columns."""
    n, L = lay.free.shape
    sd = np.full((n, L), np.nan)
    corr = np.full((n, L, L), np.nan)

    def bars(cov, scale):
        var = np.clip(np.diag(cov), 0.0, None)
        dev = np.sqrt(var)
        with np.errstate(invalid="ignore", divide="ignore"):
            return dev * scale, cov / (dev[:, None] * dev[None, :])
    blocks = {}
    if not coupled:
        for i in range(n):
            sl = np.flatnonzero(lay.free[i])
            if not sl.size:
                continue
            H = Hl[i][np.ix_(lay.pos[sl], lay.pos[sl])]
            s2 = float(resid[i] @ resid[i]) / max(resid.shape[1] - sl.size, 1)
            sd[i, sl], corr[i][np.ix_(sl, sl)] = bars(np.linalg.pinv(H) * s2, spec.scales[sl])
        return sd, corr, blocks
    P = len(lay.cols)
    JtJ = np.zeros((P, P))
    for i in range(n):
        ent = np.flatnonzero(lay.col_of[i] >= 0)
        c = lay.col_of[i, ent]
        np.add.at(JtJ, (c[:, None], c[None, :]), Hl[i][np.ix_(ent, ent)])
    s2 = float(np.sum(resid * resid)) / max(resid.size - P, 1)
    slot_of = np.array([l for l, _, _ in lay.cols], int)
    sd_c, corr_c = bars(np.linalg.pinv(JtJ) * s2, spec.scales[slot_of])
    is_block = np.array([sl.scope == "block" for sl in spec.slots])
    for i in range(n):
        sl = np.flatnonzero(lay.free[i] & ~is_block)
        c = lay.col_of[i, lay.pos[sl]]
        sd[i, sl] = sd_c[c]
        corr[i][np.ix_(sl, sl)] = corr_c[np.ix_(c, c)]
    for l in np.flatnonzero(is_block):
        c = np.flatnonzero(slot_of == l)
        vals = np.asarray(x_cols, np.float64)[c] * spec.scales[l]
        sl = spec.slots[l]
        blocks[sl.name] = dict(x=vals, sd=sd_c[c],
                               at_bounds=_near(vals, sl.lo, 1e-5, 1e-8) | _near(vals, sl.hi, 1e-5, 1e-8))
    return sd, corr, blocks


class _JointModel:
    """Per-sample model and local Jacobian of a joint fit on the GPU (joint.py:289-348)."""

    def __init__(self, params, m0, events, mz, spec, free, pos, n_loc, nb, n_per_block, spread, sig_held):
        self.params, self.m0, self.mz, self.spec = params, m0, mz, spec
        self.free, self.pos, self.n_loc, self.nb = free, pos, n_loc, nb
        self.spread, self.sig_held = spread, sig_held
        self.n = m0.shape[0]
        self.nc = n_cest_of(params)
        self.N = state_size(self.nc)
        self.is_block = np.array([s.scope == "block" for s in spec.slots])
        n_off = np.shape(events.dt)[0]
        self.n_pts = n_off
        if nb > 1:
            self.blocks = [SimEvent(*[np.asarray(a)[b * n_per_block:(b + 1) * n_per_block] for a in events])
                           for b in range(nb)]
        else:
            self.blocks = [events]
        self.dev_blocks = [DeviceEvents(e) for e in self.blocks]
        self.rows, _ = _slot_rows(spec, self.nc)
        # several blocks: every (sample, block) pair is one voxel of an uneven plan whose tables are the
        # blocks, so that one launch covers all blocks (the blocks of a few samples would not fill the GPU)
        # and with a B0 spread every isochromat is one such voxel too (the spread's nodes would otherwise run
        # one after another inside each chain)
        self.merged = None
        self.nodes = spread.nodes_weights() if spread is not None else (np.zeros(1), np.ones(1))
        if nb > 1 or spread is not None:
            from .uneven import _Plan
            nn = self.nodes[0].size
            self.merged = _Plan(self.nc, self.blocks,
                                np.repeat(np.tile(np.arange(nb, dtype=np.int32), self.n), nn), int(mz))
        self.mslot = next((l for l, s in enumerate(spec.slots) if s.field == "m_start"), None)
        self.sslot = next((l for l, s in enumerate(spec.slots) if s.field == "b0_spread"), None)

    def _effective(self, loc, b):
        """Per-sample params, start state, width and field seeds for block b (joint.py:120-138)."""
        spec = self.spec
        L = spec.n
        eff = np.where(self.free, loc[:, [self.pos[l] + (b if self.is_block[l] else 0) for l in range(L)]] *
                       spec.scales, self.carried_in[:, :L])
        upd = {}
        seeds = np.zeros((L, self.n))
        for l, s in enumerate(spec.slots):
            if s.field in PSEUDO:
                continue
            cur = np.array(upd.get(s.field, np.asarray(getattr(self.params, s.field), np.float64)), copy=True)
            old = cur if s.index is None else cur[:, s.index]
            new = eff[:, l] if s.mode == "value" else (old * eff[:, l] if s.mode == "factor" else old + eff[:, l])
            seeds[l] = np.where(self.free[:, l], s.scale * (old if s.mode == "factor" else 1.0), 0.0)
            if s.index is None:
                cur = new
            else:
                cur[:, s.index] = new
            upd[s.field] = cur
        q = self.params._replace(**upd)
        m = self.m0.copy()
        dm0 = np.zeros((L, self.n, self.N))
        if self.mslot is not None:
            ms = spec.slots[self.mslot]
            mv = eff[:, self.mslot]
            fr = self.free[:, self.mslot]
            ist = np.stack([initial_state(SimParams(*[np.asarray(v)[i] for v in q])) for i in range(self.n)])
            rebuilt = ist * mv[:, None] if ms.mode == "value" else self.m0 * mv[:, None]
            m = np.where(fr[:, None], rebuilt, self.m0)
            base_m = ist if ms.mode == "value" else self.m0
            dm0[self.mslot] = np.where(fr[:, None], base_m * ms.scale, 0.0)
            if ms.mode == "value":                     # the rebuilt state follows the pools' f
                nc = self.nc
                for l, s in enumerate(spec.slots):
                    if s.field in ("water_f", "cest_f", "mt_f"):
                        qi = {"water_f": 2 * (1 + nc), "mt_f": 3 * (1 + nc)}.get(s.field)
                        if s.field == "cest_f":
                            qi = 2 * (1 + nc) + 1 + int(s.index)
                        dm0[l, :, qi] += np.where(fr, mv * seeds[l], 0.0)
        sig = self.sig_held
        if self.sslot is not None:
            sig = np.where(self.free[:, self.sslot], eff[:, self.sslot], self.sig_held)
            seeds[self.sslot] = np.where(self.free[:, self.sslot], spec.slots[self.sslot].scale, 0.0)
        return q, m, sig, seeds, dm0

    def _evaluate_merged(self, loc, need_jac):
        """evaluate() in one launch: voxel ((i nb + b) nn + j) is sample i seen through block b at
        isochromat j (b0_inhom + sigma u_j / (gamma b0 / 2 pi), weight w_j; spread.py:77-106), and Z is the
        weighted sum over the isochromats in node order, as the kernel's own node loop forms it. The
        tangent of the spread width becomes a b0_inhom tangent seeded with u_j / (gamma b0 / 2 pi)."""
        torch = _lib.torch_cuda()
        L, n, nb, N = self.spec.n, self.n, self.nb, self.N
        u, wts = self.nodes
        nn = u.size
        Lay = lambda name: field_row(name, None, self.nc)
        row_b0i = Lay("b0_inhom")
        per = [self._effective(loc, b) for b in range(nb)]
        nf = 13 + 5 * self.nc
        P = np.empty((nf, n, nb, nn))
        M = np.empty((n, nb, nn, N))
        seeds = np.zeros((L, n, nb, nn))
        dm0 = np.zeros((L, n, nb, nn, N)) if self.mslot is not None else None
        for b, (q, m, sig, sd, dm) in enumerate(per):
            pk = pack_params(q, n)
            g = (1.0 / 6.283185307179586) * (pk[Lay("gamma")] * pk[Lay("b0")])   # Hz per ppm, as the kernel forms it
            sg = np.broadcast_to(np.asarray(sig if sig is not None else 0.0, np.float64), (n,))
            for j in range(nn):
                P[:, :, b, j] = pk
                P[row_b0i, :, b, j] = pk[row_b0i] + (u[j] * sg) / g
                M[:, b, j] = m
                seeds[:, :, b, j] = sd
                if self.sslot is not None:
                    seeds[self.sslot, :, b, j] = sd[self.sslot] * u[j] / g
                if dm0 is not None:
                    dm0[:, :, b, j] = dm
        pdev = _device(P.reshape(nf, n * nb * nn))
        mdev = _device(M.reshape(n * nb * nn, N))
        plan = self.merged
        n_per = self.n_pts // nb

        def node_sum(a):                 # (..., n, nb, nn, n_per) -> weighted sum over nn, node order
            acc = wts[0] * a[..., 0, :]
            for j in range(1, nn):
                acc = acc + wts[j] * a[..., j, :]
            return acc
        if not need_jac:
            z = plan.run(pdev, mdev).cpu().numpy().reshape(n, nb, nn, n_per)
            return (node_sum(z) if nn > 1 else z[:, :, 0]).reshape(n, nb * n_per), None
        tg = _lib.Tangents()
        tg.n_tangents = L
        for l in range(L):
            r = self.rows[l]
            tg.field_row[l] = (_lib.SEED_NONE if r == _lib.SLOT_M_START else
                               (row_b0i if r == _lib.SLOT_SPREAD_SIGMA else r))
        dseed = _device(seeds.reshape(L, n * nb * nn))
        ddm0 = _device(dm0.reshape(L, n * nb * nn, N)) if dm0 is not None else None
        tg.d_seed = dseed.data_ptr()
        tg.d_dm0 = None if ddm0 is None else ddm0.data_ptr()
        jz = torch.empty((L, plan.n_chains), dtype=torch.float64, device="cuda")
        z = plan.run(pdev, mdev, tg, jz).cpu().numpy().reshape(n, nb, nn, n_per)
        jr = jz.cpu().numpy().reshape(L, n, nb, nn, n_per)
        Z = node_sum(z) if nn > 1 else z[:, :, 0]
        Jn = node_sum(jr) if nn > 1 else jr[:, :, :, 0]
        J = np.zeros((n, self.n_pts, self.n_loc))
        for l in range(L):
            for b in range(nb):
                J[:, b * n_per:(b + 1) * n_per, self.pos[l] + (b if self.is_block[l] else 0)] = Jn[l, :, b, :]
        return Z.reshape(n, nb * n_per), J

    def evaluate(self, loc, need_jac=True):
        """Z (n, n_pts) and, with need_jac, the local Jacobian (n, n_pts, n_loc)."""
        torch = _lib.torch_cuda()
        if self.merged is not None:
            return self._evaluate_merged(loc, need_jac)
        L = self.spec.n
        Z = np.empty((self.n, self.n_pts))
        J = np.zeros((self.n, self.n_pts, self.n_loc)) if need_jac else None
        for b, dev_ev in enumerate(self.dev_blocks):
            q, m, sig, seeds, dm0 = self._effective(loc, b)
            rows = slice(b * dev_ev.n_offsets, (b + 1) * dev_ev.n_offsets)
            pdev = _device(pack_params(q, self.n))
            mdev = _device(m)
            pr = problem(self.n, dev_ev.n_offsets, dev_ev.n_events, self.nc, int(self.mz), _lib.F64)
            sp, keep = (None, None)
            if self.spread is not None:
                u, w = self.spread.nodes_weights()
                sdev = _device(np.broadcast_to(np.asarray(sig, np.float64), (self.n,)))
                sp, keep = _lib.spread_struct(u, w, sdev)
            z = torch.empty((self.n, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
            if need_jac:
                jz = torch.empty((L, self.n, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
                tg = _lib.Tangents()
                tg.n_tangents = L
                for l in range(L):
                    tg.field_row[l] = (_lib.SEED_NONE if self.rows[l] == _lib.SLOT_M_START else self.rows[l])
                sdev_seed = _device(seeds)
                ddm0 = _device(dm0) if self.mslot is not None else None
                tg.d_seed = sdev_seed.data_ptr()
                tg.d_dm0 = None if ddm0 is None else ddm0.data_ptr()
                _lib.check(_lib.lib().bmc_simulate_jvp(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev), sp, tg,
                                                       _lib.ptr(z), _lib.ptr(jz), _lib.stream_handle()))
                jl = jz.cpu().numpy()
                for l in range(L):
                    J[:, rows, self.pos[l] + (b if self.is_block[l] else 0)] = jl[l]
            else:
                _lib.check(_lib.lib().bmc_simulate(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev), sp,
                                                   _lib.ptr(z), _lib.stream_handle()))
            Z[:, rows] = z.cpu().numpy()
            del keep
        return Z, J


def _joint_solve(Hl, gl, col_of, shared, P, lam, keep=None):
    """Solve (H + lam (diag H + 1e-9 I)) d = -g for the joint columns, H = sum_i G_i^T Hl_i G_i.

    `col_of[i]` maps sample i's local entries to joint columns (-1 = not a column). Columns used by
    one sample only are eliminated per sample (block diagonal); the `shared` columns by the Schur
    complement. The same linear system as joint.py:149-162's dense solve."""
    n = Hl.shape[0]
    shared = np.asarray(sorted(shared), int)
    S = shared.size
    sidx = {c: k for k, c in enumerate(shared)}
    H_ss = np.zeros((S, S))
    g_s = np.zeros(S)
    blocks = []
    # diagonal of the full H first (the damping uses it)
    diag = np.zeros(P)
    g = np.zeros(P)
    for i in range(n):
        cols = col_of[i]
        use = np.flatnonzero(cols >= 0)
        c = cols[use]
        np.add.at(diag, c, np.diag(Hl[i])[use])
        np.add.at(g, c, gl[i][use])
    if keep is not None:
        g = g * keep
    for i in range(n):
        cols = col_of[i]
        use = np.flatnonzero(cols >= 0)
        c = cols[use]
        Hi = Hl[i][np.ix_(use, use)]
        priv = np.array([cc not in sidx for cc in c], bool)
        blocks.append((c, Hi, priv))
    # assemble: private block per sample, coupling to shared, shared block
    sol = np.zeros(P)
    Ainv_data = []
    for i, (c, Hi, priv) in enumerate(blocks):
        ks = keep[c] if keep is not None else np.ones(c.size)
        Hi = Hi * ks[:, None] * ks[None, :]
        cp, cs = c[priv], c[~priv]
        App = Hi[np.ix_(priv, priv)] + lam * np.diag(diag[cp] * (ks[priv] if keep is not None else 1.0) + 1e-9)
        if keep is not None:
            App = App + np.diag(1.0 - ks[priv]) * (1.0 + lam)
        Aps = Hi[np.ix_(priv, ~priv)]
        si = np.array([sidx[x] for x in cs], int)
        if S:
            np.add.at(H_ss, np.ix_(si, si), Hi[np.ix_(~priv, ~priv)])
        if cp.size:
            Y = np.linalg.solve(App, np.concatenate([Aps, -g[cp][:, None]], axis=1)) if cp.size else None
            Ainv_data.append((cp, si, App, Aps, Y))
            if S and si.size:
                np.add.at(H_ss, np.ix_(si, si), -Aps.T @ Y[:, :-1])
                np.add.at(g_s, si, -(Aps.T @ Y[:, -1]))
        else:
            Ainv_data.append((cp, si, None, None, None))
    if S:
        ks = keep[shared] if keep is not None else np.ones(S)
        Ass = H_ss + lam * np.diag(diag[shared] * ks + 1e-9)
        if keep is not None:
            Ass = Ass + np.diag(1.0 - ks) * (1.0 + lam)
        ds = np.linalg.solve(Ass, -g[shared] + g_s)
        sol[shared] = ds
    for cp, si, App, Aps, Y in Ainv_data:
        if cp.size:
            rhs = -g[cp] - (Aps @ sol[shared[si]] if (S and si.size) else 0.0)
            sol[cp] = np.linalg.solve(App, rhs)
    return sol


def fit_joint(experiment: Experiment, spec: FitSpec, z_meas, n_iter=30, x0_phys=None, n_per_block=None,
              max_chunk=None, lam0=1e-2, callback=None, spread=None, block_jacobian="full", stop_lam=None,
              active_bounds=False, keep_jacobian=False, _internals=False):
    """Fit every sample at once: shared, per-block and partly free values (joint.py:165-453)."""
    z = np.atleast_2d(np.asarray(z_meas, np.float64))
    n, n_pts = z.shape
    params = experiment.params
    if n_samples(params) is None:
        params = tile_params(params, n)
    if n_samples(params) != n:
        raise ValueError(f"params carry {n_samples(params)} samples, z_meas {n}")
    params = SimParams(*[np.asarray(v) for v in params])
    m0 = np.asarray(experiment.m0, np.float64)
    if m0.ndim == 1:
        m0 = np.broadcast_to(m0, (n,) + m0.shape).copy()
    events, mz = experiment.events, experiment.mz_loc
    unknown = [s.name for s in spec.slots if s.field not in PSEUDO and s.field not in SimParams._fields]
    if unknown:
        raise ValueError(f"{unknown}: not a SimParams field nor one of {PSEUDO}")
    l_sp = [l for l, s in enumerate(spec.slots) if s.field == "b0_spread"]
    if l_sp and spread is None:
        raise ValueError(f"{[spec.slots[l].name for l in l_sp]}: b0_spread needs fit_joint(..., spread=B0Spread(...))")
    if len(l_sp) > 1:
        raise ValueError(f"{[spec.slots[l].name for l in l_sp]}: one b0_spread slot at most")
    sig_held = None if spread is None else np.broadcast_to(np.asarray(spread.sigma_hz, np.float64), (n,)).copy()
    if block_jacobian not in ("full", "split"):
        raise ValueError(f"block_jacobian {block_jacobian!r}; use 'full' or 'split'")
    blocked = any(s.scope == "block" for s in spec.slots)
    if blocked and (not n_per_block or n_pts % n_per_block):
        raise ValueError(f"a per-block value needs n_per_block dividing the {n_pts} offsets (got {n_per_block})")
    nb = n_pts // n_per_block if blocked else 1
    lay = _columns(spec, n, nb)
    free, pos, n_loc, cols, col_of = lay.free, lay.pos, lay.n_loc, lay.cols, lay.col_of
    P = len(cols)
    L = spec.n
    scales = spec.scales
    is_block = np.array([s.scope == "block" for s in spec.slots])
    carried = _carried(params, m0, spec, sig_held if sig_held is not None else np.zeros(n))
    X0 = (np.broadcast_to(spec.x0_phys, free.shape) if x0_phys is None else np.asarray(x0_phys, float))
    if X0.shape != free.shape:
        raise ValueError(f"x0_phys has shape {X0.shape}, expected {free.shape} (samples, parameters)")
    X0 = np.where(free, X0, carried)

    model = _JointModel(params, m0, events, mz, spec, free, pos, n_loc, nb, n_per_block, spread,
                        sig_held if sig_held is not None else np.zeros(n))
    model.carried_in = carried
    i_ent, j_ent = np.nonzero(col_of >= 0)
    c_ent = col_of[i_ent, j_ent]

    def locs(x):
        """Every sample's local vector for the joint vector x (0 where the entry is held)."""
        loc = np.zeros((n, n_loc))
        loc[i_ent, j_ent] = np.asarray(x)[c_ent]
        return loc

    def resid(x):
        return (model.evaluate(locs(x), need_jac=False)[0] - z).reshape(-1)

    def jac(x):
        """The dense joint Jacobian (points, columns): each sample's local columns placed at their joint
        columns (a sample's entries map to distinct columns)."""
        Zm, Jl = model.evaluate(locs(x))
        J = np.zeros((n, n_pts, P))
        J[i_ent, :, c_ent] = Jl[i_ent, :, j_ent]
        return J.reshape(-1, P)

    x_start = np.asarray([X0[who[0], l] / scales[l] for l, who, _ in cols], np.float64)
    if _internals:
        return dict(resid=resid, jac=jac, x0=x_start, cols=cols, locs=locs, model=model)

    coupled = any(s.scope in ("shared", "block") for s in spec.slots)
    if not coupled and (stop_lam is not None or active_bounds or keep_jacobian):
        raise ValueError("stop_lam, active_bounds and keep_jacobian apply to a coupled fit (a shared or "
                         "per-block value); without one every sample has its own damping, as in `fit`")
    nan_steps = 0
    if not coupled:
        rows, modes = _slot_rows(spec, model.nc)
        lo, hi = spec.lo_phys / scales, spec.hi_phys / scales
        hold = None if free.all() else free.astype(np.float64)
        X0s = X0 / scales
        chunk = max_chunk or n
        xs, cs = [], []
        for a in range(0, n, chunk):
            b = min(a + chunk, n)
            sub = SimParams(*[np.asarray(v)[a:b] for v in params])
            x, c = _lm_device(sub, events, m0[a:b], mz, rows, modes, scales, lo, hi, z[a:b], X0s[a:b], n_iter,
                              lam0, 0, None if hold is None else hold[a:b], spread,
                              None if sig_held is None else sig_held[a:b])
            xs.append(x)
            cs.append(c)
        loc = np.concatenate(xs)
        cost = np.concatenate(cs).sum(axis=0)
    else:
        col_slot = np.array([l for l, _, _ in cols], int)
        col_scale = scales[col_slot]
        lo = spec.lo_phys[col_slot] / col_scale
        hi = spec.hi_phys[col_slot] / col_scale
        shared_cols = [p for p, (l, who, b) in enumerate(cols) if len(who) > 1 or b >= 0]
        x = x_start.copy()
        lam, cost = float(lam0), []
        kept = None
        for it in range(n_iter):
            if kept is None:
                Zm, Jl = model.evaluate(locs(x))
                r = (Zm - z)
                finite = bool(np.all(np.isfinite(Jl)))
            else:
                (r, Jl), finite = kept, True
            c = float(np.sum(r * r))
            if finite:
                Hl = np.einsum("inj,ink->ijk", Jl, Jl)
                gl = np.einsum("inj,in->ij", Jl, r)
                keep = None
                if active_bounds:
                    g_full = np.bincount(c_ent, weights=gl[i_ent, j_ent], minlength=P)
                    keep = np.where(((x <= lo) & (g_full > 0)) | ((x >= hi) & (g_full < 0)), 0.0, 1.0)
                d = _joint_solve(Hl, gl, col_of, shared_cols, P, lam, keep)
                xn = np.clip(x + d, lo, hi)
                cn = float(np.sum(resid(xn) ** 2))
                better = cn < c
                kept = (r, Jl) if keep_jacobian and not better else None
                x = xn if better else x
                lam = lam * 0.5 if better else lam * 3.0
                cost.append(cn if better else c)
            else:
                nan_steps += 1
                lam = lam * 3.0
                cost.append(c)
                kept = None
            if callback is not None:
                callback(it, cost[-1])
            if stop_lam is not None and lam > stop_lam:
                break
        loc = locs(x)
        cost = np.asarray(cost)

    X = np.where(free, loc[:, pos] * scales, carried)
    Zf, Jl = model.evaluate(loc)
    r_all = Zf - z
    sd, corr, blocks = _error_bars(np.einsum("inj,ink->ijk", Jl, Jl), r_all, lay, spec, coupled,
                                   x if coupled else None)
    X[:, is_block] = np.nan
    X0 = np.where(is_block[None, :], np.nan, X0)
    free = free & ~is_block[None, :]
    return FitResult(X, Zf, z, spec, n_per_block, free=free, sd=sd, corr=corr, x0=X0, cost=cost,
                     nan_steps=nan_steps, blocks=blocks or None)
