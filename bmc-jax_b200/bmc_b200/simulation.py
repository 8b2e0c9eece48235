"""The forward model: BMC-JAX's `bmc_jax.simulation` API on the B200 kernels.

Same names, arguments, layouts and error messages as the reference (simulation/params.py,
events.py, simulate.py, voxels.py, spread.py); the arrays are NumPy on the host. Every simulation
runs in libbmc_b200.so (one GPU thread per (voxel, offset) chain, the whole event table per
thread); there is no CPU path.

Precision: the propagation runs in float64 by default (B200 executes float64 at half its float32
rate, and float64 agrees with the reference's x64 path to ~1e-12); `settings.use_x64(False)` selects
the float32 kernel for forward simulations. Tangents and fits are always float64.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, List, NamedTuple, Optional

import numpy as np

from . import _lib, settings

__all__ = ["SimParams", "SimEvent", "EventType", "to_sim_params", "initial_state", "cast_params",
           "cast_events", "pad_events", "repeat_events", "tile_params", "stack_params", "extract_z_spectra",
           "simulate_spectrum", "simulate_voxels", "B0Spread", "simulate_spectrum_spread", "state_size",
           "SHAPES"]


class SimParams(NamedTuple):
    """BMC parameters, field for field the reference SimParams (simulation/params.py:18-49).

    Scalars per sample, `cest_*` of length n_cest; batched params carry a leading sample axis."""
    water_r1: Any
    water_r2: Any
    water_f: Any
    cest_k: Any
    cest_f: Any
    cest_dw: Any
    cest_r1: Any
    cest_r2: Any
    mt_k: Any
    mt_f: Any
    mt_dw: Any
    mt_r1: Any
    mt_r2: Any
    mt_lineshape: Any
    b0: Any
    gamma: Any
    b0_inhom: Any
    rel_b1: Any


class EventType:
    """Event type codes (simulation/events.py:12-18)."""
    DELAY = 0
    RF_PULSE = 1
    GRADIENT = 2
    ADC = 3
    SPOILER = 4


class SimEvent(NamedTuple):
    """The event table, each field (n_offsets, n_events) (simulation/events.py:20-32)."""
    type: Any
    dt: Any
    rf_amp: Any
    rf_phase: Any
    rf_freq: Any
    adc_idx: Any


POOL_FIELDS = ("cest_k", "cest_f", "cest_dw", "cest_r1", "cest_r2")


def n_cest_of(p: SimParams) -> int:
    s = np.shape(p.cest_k)
    return int(s[-1]) if len(s) else 0


def state_size(n_cest: int) -> int:
    """3 (1 + n_cest) + 1: x, y, z of water and each CEST pool, then MT z (matrix.py:216-219)."""
    return 3 * (1 + n_cest) + 1


# ------------------------------------------------------------------------------------------------
# parameters (simulation/params.py)
# ------------------------------------------------------------------------------------------------
def to_sim_params(params: Any, max_cest_pools: Optional[int] = None) -> SimParams:
    """A Pulseq-CEST style object (water_pool, cest_pools, mt_pool, system) -> SimParams, pools
    zero-padded to `max_cest_pools` (simulation/params.py:51-152). Duck-typed, like the reference."""
    f = lambda v: np.asarray(v, dtype=float)
    pools = list(params.cest_pools)
    target = max_cest_pools if max_cest_pools is not None else len(pools)
    if target < len(pools):
        raise ValueError(f"max_cest_pools ({max_cest_pools}) is smaller than actual number of pools ({len(pools)})")
    pad = target - len(pools)
    col = lambda name: f([getattr(p, name) for p in pools] + [0.0] * pad)
    mt = params.mt_pool
    if mt is not None:
        ls = {"lorentzian": 1, "superlorentzian": 2}.get(str(mt.lineshape).lower(), 0)
        mtv = (f(mt.k), f(mt.f), f(mt.dw), f(mt.r1), f(mt.r2), np.asarray(ls))
    else:
        mtv = (f(0.0), f(0.0), f(0.0), f(0.0), f(1.0), np.asarray(0))
    s = params.system
    return SimParams(f(params.water_pool.r1), f(params.water_pool.r2), f(params.water_pool.f),
                     col("k"), col("f"), col("dw"), col("r1"), col("r2"), *mtv,
                     f(s.b0), f(s.gamma), f(s.b0_inhom), f(s.rel_b1))


def initial_state(jax_params: SimParams, m_start: float = 1.0) -> np.ndarray:
    """M0: water, CEST and MT z set to their fractions, all times m_start (params.py:154-212)."""
    p = jax_params
    nc = n_cest_of(p)
    n = 1 + nc
    dtype = np.result_type(np.asarray(p.water_f).dtype, np.float32)
    M = np.zeros(3 * n + 1, dtype)
    M[2 * n] = p.water_f
    M[2 * n + 1:3 * n] = np.asarray(p.cest_f).reshape(nc)
    M[3 * n] = p.mt_f
    if m_start != 1.0:
        M = M * m_start
    return M


def cast_params(params: SimParams, dtype) -> SimParams:
    """Every physical field to `dtype`; the lineshape code stays an integer (params.py:215-228)."""
    return SimParams(**{k: (np.asarray(getattr(params, k)) if k == "mt_lineshape"
                            else np.asarray(getattr(params, k)).astype(dtype)) for k in SimParams._fields})


def tile_params(params: SimParams, n_voxels: int) -> SimParams:
    """One tissue repeated into a batch of n_voxels (voxels.py:74-83)."""
    return SimParams(*[np.broadcast_to(np.asarray(v), (n_voxels,) + np.shape(v)) for v in params])


def stack_params(params_list: List[SimParams]) -> SimParams:
    """Per-voxel SimParams into one batch (voxels.py:47-71)."""
    if not params_list:
        raise ValueError("params_list is empty")
    return SimParams(*[np.stack([np.asarray(getattr(p, k)) for p in params_list]) for k in SimParams._fields])


def extract_z_spectra(trajectory, water_z_index: int):
    """Water Mz of every final state (voxels.py:135-151)."""
    return np.asarray(trajectory)[..., water_z_index]


# ------------------------------------------------------------------------------------------------
# events (simulation/events.py)
# ------------------------------------------------------------------------------------------------
def pad_events(events: SimEvent, width: int) -> SimEvent:
    """Front-pad to `width` events with zero-duration DELAYs, a true no-op (events.py:34-91)."""
    n_offsets, n_events = np.shape(events.dt)
    if width < n_events:
        raise ValueError(f"cannot pad {n_events} events down to {width}")
    if width == n_events:
        return events
    k = width - n_events

    def pre(leaf, fill):
        leaf = np.asarray(leaf)
        return np.concatenate([np.full((n_offsets, k), fill, leaf.dtype), leaf], axis=1)
    return SimEvent(pre(events.type, EventType.DELAY), pre(events.dt, 0.0), pre(events.rf_amp, 0.0),
                    pre(events.rf_phase, 0.0), pre(events.rf_freq, 0.0), pre(events.adc_idx, -1))


def cast_events(events: SimEvent, dtype) -> SimEvent:
    """Floating fields to `dtype` (events.py:94-103)."""
    return SimEvent(np.asarray(events.type), *[np.asarray(getattr(events, k)).astype(dtype)
                                              for k in ("dt", "rf_amp", "rf_phase", "rf_freq")],
                    np.asarray(events.adc_idx))


def repeat_events(events: SimEvent, n_reps: int) -> SimEvent:
    """The batch of offsets replicated n_reps times (events.py:106-115)."""
    return SimEvent(*[np.tile(np.asarray(a), (n_reps, 1)) for a in events])


# ------------------------------------------------------------------------------------------------
# marshalling to the C ABI
# ------------------------------------------------------------------------------------------------
def pack_params(p: SimParams, n_vox: int) -> np.ndarray:
    """SimParams (one sample or a batch of n_vox) -> the ABI layout [13 + 5 n_cest][n_vox] float64."""
    nc = n_cest_of(p)
    rows = []
    for k in SimParams._fields:
        v = np.asarray(getattr(p, k), dtype=np.float64)
        if k in POOL_FIELDS:
            v = np.broadcast_to(v, (n_vox, nc)) if v.ndim <= 1 else v
            if v.shape != (n_vox, nc):
                raise ValueError(f"{k}: shape {v.shape} for {n_vox} samples of {nc} pools")
            rows.extend(v.T)
        else:
            v = np.broadcast_to(v.reshape(-1) if v.ndim else v, (n_vox,))
            rows.append(v)
    return np.ascontiguousarray(np.stack(rows), dtype=np.float64)


def n_samples(p: SimParams) -> Optional[int]:
    """Leading batch size, or None for one sample."""
    return int(np.shape(p.water_r1)[0]) if np.ndim(p.water_r1) > 0 else None


class DeviceEvents:
    """An event table on the device (the six reference fields), kept alive for a C call."""

    def __init__(self, events: SimEvent):
        torch = _lib.torch_cuda()
        dt = np.asarray(events.dt)
        if dt.ndim != 2:
            raise ValueError(f"events must be (n_offsets, n_events), got {dt.shape}")
        self.n_offsets, self.n_events = dt.shape
        cuda = torch.device("cuda")
        as_i = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a), np.int32)).to(cuda)
        as_f = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a), np.float64)).to(cuda)
        self.t = [as_i(events.type), as_f(events.dt), as_f(events.rf_amp), as_f(events.rf_phase),
                  as_f(events.rf_freq), as_i(events.adc_idx)]
        self.struct = _lib.Events(*[x.data_ptr() for x in self.t])

    @classmethod
    def from_tensors(cls, type_, dt, amp, phase, freq, adc):
        """Wrap device tensors that already hold a table (no copy)."""
        self = cls.__new__(cls)
        self.n_offsets, self.n_events = dt.shape
        self.t = [type_, dt, amp, phase, freq, adc]
        self.struct = _lib.Events(*[x.data_ptr() for x in self.t])
        return self


def _device(a, dtype=np.float64):
    torch = _lib.torch_cuda()
    return torch.as_tensor(np.require(np.asarray(a, dtype), requirements=["C", "W"])).to(torch.device("cuda"))


def problem(n_vox, n_off, n_ev, n_cest, mz, precision=None, reset_after_adc=True):
    prec = {"f64": _lib.F64, "mixed": _lib.MIXED, "f32": _lib.F32}[settings.precision()] if precision is None \
        else precision
    return _lib.Problem(n_vox, n_off, n_ev, n_cest, mz, 1 if reset_after_adc else 0, prec, 0)


def simulate_device(pr, params_dev, dev_ev, m0_dev, out_dev, spread=None):
    """The raw call on device tensors: Z or full final states into `out_dev`."""
    sp, keep = spread if spread is not None else (None, None)
    _lib.check(_lib.lib().bmc_simulate(pr, _lib.ptr(params_dev), dev_ev.struct, _lib.ptr(m0_dev),
                                       sp, _lib.ptr(out_dev), _lib.stream_handle()))
    return keep


def _simulate(params: SimParams, events: SimEvent, M_init, mz: int, spread=None,
              precision=None) -> np.ndarray:
    torch = _lib.torch_cuda()
    nb = n_samples(params)
    nv = nb if nb is not None else 1
    nc = n_cest_of(params)
    N = state_size(nc)
    m0 = np.asarray(M_init, np.float64)
    m0 = np.broadcast_to(m0.reshape(-1, N) if m0.ndim > 1 else m0, (nv, N))
    dev_ev = DeviceEvents(events)
    pdev = _device(pack_params(params, nv))
    mdev = _device(m0)
    shape = (nv, dev_ev.n_offsets) if mz >= 0 else (nv, dev_ev.n_offsets, N)
    out = torch.empty(shape, dtype=torch.float64, device="cuda")
    pr = problem(nv, dev_ev.n_offsets, dev_ev.n_events, nc, mz, precision)
    keep = None
    sp = None
    if spread is not None:
        u, w, sigma = spread
        sdev = _device(np.broadcast_to(np.asarray(sigma, np.float64), (nv,)))
        sp = _lib.spread_struct(u, w, sdev)
    keep = simulate_device(pr, pdev, dev_ev, mdev, out, sp)
    res = out.cpu().numpy()
    del keep
    return res if nb is not None else res[0]


def _trajectory(params: SimParams, events: SimEvent, M_init) -> np.ndarray:
    torch = _lib.torch_cuda()
    nc = n_cest_of(params)
    N = state_size(nc)
    dev_ev = DeviceEvents(events)
    pdev = _device(pack_params(params, 1))
    mdev = _device(np.asarray(M_init, np.float64).reshape(1, N))
    out = torch.empty((1, dev_ev.n_offsets, dev_ev.n_events, N), dtype=torch.float64, device="cuda")
    pr = problem(1, dev_ev.n_offsets, dev_ev.n_events, nc, 0, _lib.F64)
    _lib.check(_lib.lib().bmc_simulate_trajectory(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev),
                                                  _lib.ptr(out), _lib.stream_handle()))
    return out.cpu().numpy()[0]


# ------------------------------------------------------------------------------------------------
# simulate (simulation/simulate.py, voxels.py)
# ------------------------------------------------------------------------------------------------
def simulate_spectrum(params: SimParams, events: SimEvent, M_init, return_full_trajectory: bool = True):
    """Every offset of one sample: (n_offsets, n_events, N) trajectories, or (n_offsets, N) final
    states with return_full_trajectory=False (simulate.py:134-148)."""
    if n_samples(params) is not None:
        raise ValueError("simulate_spectrum takes one sample; use simulate_voxels for a batch")
    if return_full_trajectory:
        return _trajectory(params, events, M_init)
    return _simulate(params, events, M_init, -1)


def simulate_voxels(params_batch: SimParams, events: SimEvent, M_init_batch, return_full_trajectory: bool = False):
    """Many voxels against one shared event table: (n_voxels, n_offsets, N) (voxels.py:89-129)."""
    if n_samples(params_batch) is None:
        raise ValueError("simulate_voxels needs params with a leading voxel axis")
    if return_full_trajectory:
        return np.stack([_trajectory(SimParams(*[np.asarray(v)[i] for v in params_batch]), events,
                                     np.asarray(M_init_batch)[i]) for i in range(n_samples(params_batch))])
    return _simulate(params_batch, events, M_init_batch, -1)


def simulate_z(params: SimParams, events: SimEvent, M_init, mz: int, precision=None) -> np.ndarray:
    """Only state[mz] of every offset (what Experiment.simulate and fitting read)."""
    return _simulate(params, events, M_init, int(mz), precision=precision)


# ------------------------------------------------------------------------------------------------
# B0 spread (simulation/spread.py)
# ------------------------------------------------------------------------------------------------
SHAPES = ("gauss", "lorentz")


@dataclass(frozen=True)
class B0Spread:
    """The distribution of the field offset inside a sample (spread.py:38-74)."""
    sigma_hz: Any = 0.0
    shape: str = "gauss"
    nodes: int = 5
    cut: float = 20.0

    def __post_init__(self):
        if self.shape not in SHAPES:
            raise ValueError(f"B0Spread shape {self.shape!r}; use one of {SHAPES}")
        if int(self.nodes) < 1:
            raise ValueError(f"B0Spread nodes {self.nodes}: at least 1")
        if self.shape == "lorentz" and not self.cut > 0:
            raise ValueError(f"B0Spread cut {self.cut}: must be positive")

    def nodes_weights(self):
        """(u, w): offsets in units of sigma, weights summing to 1 (numpy, float64)."""
        if self.shape == "gauss":
            u, w = np.polynomial.hermite_e.hermegauss(int(self.nodes))
        else:
            t, w = np.polynomial.legendre.leggauss(int(self.nodes))
            u = np.tan(t * np.arctan(self.cut))
        return u, w / w.sum()


def simulate_spectrum_spread(params, events, M_init, sigma_hz, spread: B0Spread):
    """(n_offsets, N): the weighted mean over the spread's isochromats (spread.py:77-106)."""
    u, w = spread.nodes_weights()
    return _simulate(params, events, M_init, -1, spread=(u, w, sigma_hz))
