"""CPU oracle for the BMC-JAX hot path -- TEST INFRASTRUCTURE, never part of the product.

A float64 NumPy restatement of the reference algorithm, written from its source (file:line below,
paths relative to the BMC-JAX project). Only `tests/`, `__graft_entry__.smoke()` and the CPU legs of
`bench.py` may import it, and only as the checker or the timed CPU baseline.

Pinning. The reference needs JAX, which cannot be installed here, so the reference is executed on
a NumPy stand-in for the JAX subset it uses (tests/golden/_jaxshim, script tests/golden/make_golden.py)
and its outputs are committed as golden vectors; tests/test_oracle_golden.py checks this module
against them. The reference's own physics invariants (tests/test_solver.py) and its README
quick-start answer (README.md:62-94) are checked as well.

What is restated:
  super_lorentzian / lorentzian       simulation/matrix.py:25-81
  bmc_system (A, C)                   simulation/matrix.py:83-295
  propagate                           simulation/expm.py:86-112 (float64 library path: an accurate expm)
  simulate_chain                      simulation/simulate.py:22-132
  simulate_spectrum / _voxels         simulation/simulate.py:134-148, simulation/voxels.py:89-129
  spread_nodes / simulate_spread      simulation/spread.py:38-106
  initial_state                       simulation/params.py:154-212
  cw_saturation                       sequences/saturation.py:28-84
  pad_events / stack_events           simulation/events.py:34-91, fitting/experiment.py:101-141
  jacobian (forward mode)             the derivative jax.jacfwd takes (fitting/lm.py:39)
  levenberg_marquardt                 fitting/lm.py:20-67
  lm_trial                            fitting/joint.py:149-162

The Jacobian is exact forward mode: each parameter's derivative of the system matrix comes from a
complex step through `bmc_system` (written to be complex-analytic), and each time step's tangent
from the Frechet derivative of the matrix exponential (scipy.linalg.expm_frechet).
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import NamedTuple

import numpy as np
import scipy.linalg as sla

# event types, simulation/events.py:12-18
DELAY, RF_PULSE, GRADIENT, ADC, SPOILER = 0, 1, 2, 3, 4

GAMMA_RAD_PER_S_UT = 267.5153          # sequences/saturation.py:14
GAMMA_HZ_PER_T = 42.5764e6             # sequences/saturation.py:16

SCALAR_FIELDS = ("water_r1", "water_r2", "water_f", "mt_k", "mt_f", "mt_dw", "mt_r1", "mt_r2",
                 "mt_lineshape", "b0", "gamma", "b0_inhom", "rel_b1")
POOL_FIELDS = ("cest_k", "cest_f", "cest_dw", "cest_r1", "cest_r2")
# SimParams field order, simulation/params.py:18-49
FIELDS = ("water_r1", "water_r2", "water_f", "cest_k", "cest_f", "cest_dw", "cest_r1", "cest_r2",
          "mt_k", "mt_f", "mt_dw", "mt_r1", "mt_r2", "mt_lineshape", "b0", "gamma", "b0_inhom",
          "rel_b1")


class Params(NamedTuple):
    """Same fields, order and meaning as the reference SimParams (simulation/params.py:18-49)."""
    water_r1: np.ndarray
    water_r2: np.ndarray
    water_f: np.ndarray
    cest_k: np.ndarray
    cest_f: np.ndarray
    cest_dw: np.ndarray
    cest_r1: np.ndarray
    cest_r2: np.ndarray
    mt_k: np.ndarray
    mt_f: np.ndarray
    mt_dw: np.ndarray
    mt_r1: np.ndarray
    mt_r2: np.ndarray
    mt_lineshape: np.ndarray
    b0: np.ndarray
    gamma: np.ndarray
    b0_inhom: np.ndarray
    rel_b1: np.ndarray


class Events(NamedTuple):
    """Same fields as the reference SimEvent (simulation/events.py:20-32); each (n_offsets, n_events)."""
    type: np.ndarray
    dt: np.ndarray
    rf_amp: np.ndarray
    rf_phase: np.ndarray
    rf_freq: np.ndarray
    adc_idx: np.ndarray


def make_params(water_r1, water_r2, cest_k=(), cest_f=(), cest_dw=(), cest_r1=(), cest_r2=(),
                water_f=1.0, mt=None, b0=3.0, gamma=GAMMA_RAD_PER_S_UT, b0_inhom=0.0, rel_b1=1.0):
    """One sample's Params. `mt` = dict(k, f, dw, r1, r2, lineshape) or None (reference defaults
    when absent: zeros, r2 = 1, lineshape 0, simulation/params.py:117-125)."""
    a = lambda v: np.asarray(v, np.float64)
    if mt is None:
        mt = dict(k=0.0, f=0.0, dw=0.0, r1=0.0, r2=1.0, lineshape=0)
    return Params(a(water_r1), a(water_r2), a(water_f), a(cest_k), a(cest_f), a(cest_dw), a(cest_r1),
                  a(cest_r2), a(mt["k"]), a(mt["f"]), a(mt["dw"]), a(mt["r1"]), a(mt["r2"]),
                  np.asarray(mt["lineshape"], np.int64), a(b0), a(gamma), a(b0_inhom), a(rel_b1))


def n_cest_of(p: Params) -> int:
    return int(np.shape(p.cest_k)[-1]) if np.ndim(p.cest_k) else 0


def state_size(n_cest: int) -> int:
    """N = 3 (1 + n_cest) + 1: x, y, z of water and every CEST pool, then MT z (matrix.py:216-219)."""
    return 3 * (1 + n_cest) + 1


def mz_loc(n_cest: int) -> int:
    """Index of water Mz, io/parameters/parameters.py:56-67."""
    return 2 * (1 + n_cest)


def sample(p: Params, i: int) -> Params:
    """Sample i of a batched Params (leading axis)."""
    return Params(*[np.asarray(v)[i] for v in p])


def tile(p: Params, n: int) -> Params:
    return Params(*[np.broadcast_to(np.asarray(v), (n,) + np.shape(v)).copy() for v in p])


# ------------------------------------------------------------------------------------------------
# lineshapes (matrix.py:25-81). Written so that a complex step through them gives the derivative:
# `_rabs` is |x| for a real-valued quantity, continued analytically; comparisons use the real part.
# ------------------------------------------------------------------------------------------------
_SL_U = np.linspace(0.0, 1.0, 101)
_SL_T = np.maximum(np.abs(3.0 * _SL_U ** 2 - 1.0), 1e-6)      # |3u^2-1| floored at 1e-6
_SL_DU = 0.01


def _rabs(x):
    return np.where(np.real(x) >= 0, x, -x)


def _sl_direct(delta, t2):
    arg = delta * t2 / _SL_T
    integrand = np.sqrt(2.0 / np.pi) * t2 / _SL_T * np.exp(-2.0 * arg ** 2)
    return np.sum(integrand) * np.pi * _SL_DU


def super_lorentzian(delta, t2, w0):
    """Super-Lorentzian g(delta) [s]; a cubic Hermite bridge inside |delta| < w0 (matrix.py:40-68)."""
    if np.real(_rabs(delta)) >= np.real(w0):
        return _sl_direct(delta, t2)
    px = [-300.0 - w0, -100.0 - w0, 100.0 + w0, 300.0 + w0]
    py0, py1, py2, py3 = (_sl_direct(v, t2) for v in px)
    d0y = 30.0 * (py1 - py0)
    d1y = 30.0 * (py3 - py2)
    c = _rabs((delta - px[1] + 1.0) / (px[2] - px[1] + 1.0))
    h0 = 2 * c ** 3 - 3 * c ** 2 + 1
    h1 = -2 * c ** 3 + 3 * c ** 2
    h2 = c ** 3 - 2 * c ** 2 + c
    h3 = c ** 3 - c ** 2
    return h0 * py1 + h1 * py2 + h2 * d0y + h3 * d1y


def lorentzian(delta, t2):
    return t2 / (1.0 + (delta * t2) ** 2)


# ------------------------------------------------------------------------------------------------
# the system matrix (matrix.py:83-295)
# ------------------------------------------------------------------------------------------------
def bmc_system(p: Params, rf_amp, rf_phase, rf_freq):
    """A (N x N) and C (N) of dM/dt = A M + C for one sample and one RF state.

    The state layout is the reference's: water x at 0, CEST x at 1..n, water y at n+1, CEST y after
    it, water z at 2(n+1), CEST z after it, MT z last (matrix.py:224-234)."""
    nc = n_cest_of(p)
    dtype = np.result_type(*[np.asarray(v) for v in p], rf_amp, rf_phase, rf_freq, np.float64)
    k = np.asarray(p.cest_k).reshape(nc)
    f = np.asarray(p.cest_f).reshape(nc)
    r1c = np.asarray(p.cest_r1).reshape(nc)
    r2c = np.asarray(p.cest_r2).reshape(nc)
    dwc = np.asarray(p.cest_dw).reshape(nc)
    kwc = k * f
    kwmt = p.mt_k * p.mt_f
    w1 = 2.0 * np.pi * rf_amp * p.rel_b1
    w1x, w1y = w1 * np.cos(rf_phase), w1 * np.sin(rf_phase)
    larmor = p.gamma * 1e6 * p.b0
    dw0 = larmor * p.b0_inhom * 1e-6
    eff = 2.0 * np.pi * rf_freq - dw0                   # one offset seen by every pool (matrix.py:162)
    off_c = dwc * 1e-6 * larmor - eff
    off_w = eff
    off_mt = eff - p.mt_dw * 1e-6 * larmor
    t2mt = 1.0 / p.mt_r2
    g = 0.0
    if np.real(p.mt_f) > 1e-9:                           # matrix.py:203-213
        ls = int(np.real(p.mt_lineshape))
        ls = min(max(ls, 0), 2)                          # lax.switch clamps the index
        if ls == 1:
            g = lorentzian(off_mt, t2mt)
        elif ls == 2:
            g = super_lorentzian(off_mt, t2mt, larmor * 1e-6)
    w_mt = w1 ** 2 * g if np.real(p.mt_f) > 1e-9 else 0.0

    n = 1 + nc
    N = 3 * n + 1
    A = np.zeros((N, N), dtype)
    C = np.zeros(N, dtype)
    xw, yw, zw, zm = 0, n, 2 * n, 3 * n
    ksum = np.sum(kwc)
    A[xw, xw] = -p.water_r2 - ksum
    A[xw, yw] = off_w
    A[xw, zw] = -w1y
    A[yw, yw] = -p.water_r2 - ksum
    A[yw, xw] = -off_w
    A[yw, zw] = w1x
    A[zw, zw] = -p.water_r1 - ksum - kwmt
    A[zw, yw] = -w1x
    A[zw, xw] = w1y
    for i in range(nc):
        xc, yc, zc = 1 + i, n + 1 + i, 2 * n + 1 + i
        A[xc, xc] = -r2c[i] - k[i]
        A[xc, yc] = -off_c[i]
        A[xc, zc] = -w1y
        A[yc, yc] = -r2c[i] - k[i]
        A[yc, xc] = off_c[i]
        A[yc, zc] = w1x
        A[zc, zc] = -r1c[i] - k[i]
        A[zc, xc] = w1y
        A[zc, yc] = -w1x
        A[xw, xc] = k[i]
        A[yw, yc] = k[i]
        A[zw, zc] = k[i]
        A[xc, xw] = kwc[i]
        A[yc, yw] = kwc[i]
        A[zc, zw] = kwc[i]
        C[zc] = r1c[i] * f[i]
    A[zm, zm] = -p.mt_r1 - p.mt_k - w_mt
    A[zm, zw] = kwmt
    A[zw, zm] = p.mt_k
    C[zw] = p.water_r1 * 1.0
    C[zm] = p.mt_r1 * p.mt_f
    return A, C


def augmented(A, C, dt):
    """[A C; 0 0] * dt, the homogeneous-coordinate generator (expm.py:86-112)."""
    N = A.shape[0]
    X = np.zeros((N + 1, N + 1), A.dtype)
    X[:N, :N] = A
    X[:N, N] = C
    return X * dt


def propagate(M, dt, A, C):
    """M <- first N entries of expm([A C; 0 0] dt) [M; 1]."""
    E = sla.expm(augmented(A, C, dt))
    return (E @ np.append(M, 1.0))[:-1]


def initial_state(p: Params, m_start: float = 1.0):
    """M0: z entries f (water, CEST, MT), times m_start (simulation/params.py:154-212)."""
    nc = n_cest_of(p)
    n = 1 + nc
    M = np.zeros(3 * n + 1, np.result_type(p.water_f, p.cest_f, p.mt_f, np.float64))
    M[2 * n] = p.water_f
    M[2 * n + 1:3 * n] = np.asarray(p.cest_f).reshape(nc)
    M[3 * n] = p.mt_f
    return M * m_start if m_start != 1.0 else M


# ------------------------------------------------------------------------------------------------
# the event scan (simulate.py:22-132)
# ------------------------------------------------------------------------------------------------
def _spoil(M, nc):
    out = M.copy()
    out[:2 * (1 + nc)] = 0.0                            # x and y of water and every CEST pool
    return out


def simulate_chain(p: Params, ev_row: Events, M0, reset_after_adc=True, return_trajectory=False):
    """One offset: scan over its events; returns last_M (the state after the last event, before any
    ADC reset), or the (n_events, N) trajectory of post-event states."""
    nc = n_cest_of(p)
    M = np.asarray(M0, np.float64).copy()
    last = M.copy()
    traj = []
    for j in range(len(ev_row.dt)):
        t = int(ev_row.type[j])
        dt = float(ev_row.dt[j])
        if dt > 1e-9:
            A, C = bmc_system(p, float(ev_row.rf_amp[j]), float(ev_row.rf_phase[j]), float(ev_row.rf_freq[j]))
            M = propagate(M, dt, A, C)
        if t == GRADIENT or t == SPOILER:
            M = _spoil(M, nc)
        last = M
        traj.append(M.copy())
        if t == ADC and reset_after_adc:
            M = np.asarray(M0, np.float64).copy()
    return np.array(traj) if return_trajectory else last


def event_row(ev: Events, i: int) -> Events:
    return Events(*[np.asarray(a)[i] for a in ev])


def simulate_spectrum(p: Params, ev: Events, M0):
    """(n_offsets, N): final states of every offset (simulate.py:134-148)."""
    return np.stack([simulate_chain(p, event_row(ev, i), M0) for i in range(ev.dt.shape[0])])


def simulate_voxels(pb: Params, ev: Events, M0b):
    """(n_voxels, n_offsets, N) for batched params and start states (voxels.py:89-129)."""
    return np.stack([simulate_spectrum(sample(pb, v), ev, np.asarray(M0b)[v]) for v in range(np.shape(pb.water_r1)[0])])


# ------------------------------------------------------------------------------------------------
# B0 spread (spread.py:38-106)
# ------------------------------------------------------------------------------------------------
def spread_nodes(shape="gauss", nodes=5, cut=20.0):
    """(u, w): offsets in units of sigma and weights summing to 1."""
    if shape == "gauss":
        u, w = np.polynomial.hermite_e.hermegauss(int(nodes))
    elif shape == "lorentz":
        t, w = np.polynomial.legendre.leggauss(int(nodes))
        u = np.tan(t * np.arctan(cut))
    else:
        raise ValueError(shape)
    return u, w / w.sum()


def simulate_spread(p: Params, ev: Events, M0, sigma_hz, shape="gauss", nodes=5, cut=20.0):
    """Weighted mean over isochromats at b0_inhom + sigma u / (gamma B0 / 2 pi) (spread.py:77-106)."""
    u, w = spread_nodes(shape, nodes, cut)
    hz_per_ppm = p.gamma * p.b0 / (2.0 * np.pi)
    out = 0.0
    for uj, wj in zip(u, w):
        q = p._replace(b0_inhom=p.b0_inhom + sigma_hz * uj / hz_per_ppm)
        out = out + wj * simulate_spectrum(q, ev, M0)
    return out


# ------------------------------------------------------------------------------------------------
# sequences and event tables
# ------------------------------------------------------------------------------------------------
def hz_per_ppm(b0_T):
    return GAMMA_HZ_PER_T * b0_T / 1e6


def cw_saturation(ppm, b1_uT, tsat_s, b0_T=2.8936, m0_ppm=None) -> Events:
    """One CW block then a zero-length ADC per offset (sequences/saturation.py:28-84).
    Floating fields are rounded to float32 first, as the reference builds them."""
    ppm = np.atleast_1d(np.asarray(ppm, np.float64))
    if m0_ppm is not None:
        ppm = np.concatenate([[float(m0_ppm)], ppm])
    if tsat_s < 0 or b1_uT < 0:
        raise ValueError("tsat_s and b1_uT must be >= 0")
    n = ppm.size
    amp = b1_uT * GAMMA_RAD_PER_S_UT / (2 * np.pi)
    freq = ppm * hz_per_ppm(b0_T)
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    col = lambda a, b: np.stack([np.broadcast_to(a, n), np.broadcast_to(b, n)], axis=1)
    return Events(type=col(RF_PULSE, ADC).astype(np.int32), dt=f32(col(tsat_s, 0.0)),
                  rf_amp=f32(col(amp, 0.0)), rf_phase=f32(col(0.0, 0.0)),
                  rf_freq=f32(col(freq, np.zeros(n))), adc_idx=col(-1, 0).astype(np.int32))


def pad_events(ev: Events, width: int) -> Events:
    """Front-pad with zero-duration DELAYs, a bit-exact no-op (events.py:34-91)."""
    n_off, n_ev = ev.dt.shape
    if width < n_ev:
        raise ValueError(f"cannot pad {n_ev} events down to {width}")
    k = width - n_ev
    pre = lambda a, v: np.concatenate([np.full((n_off, k), v, np.asarray(a).dtype), a], axis=1)
    return Events(pre(ev.type, DELAY), pre(ev.dt, 0.0), pre(ev.rf_amp, 0.0), pre(ev.rf_phase, 0.0),
                  pre(ev.rf_freq, 0.0), pre(ev.adc_idx, -1))


def stack_events(evs) -> Events:
    """Experiment.stack's event table: pad to the longest, concatenate offsets (experiment.py:101-141)."""
    evs = list(evs)
    if not evs:
        raise ValueError("stack needs at least one experiment")
    width = max(e.dt.shape[1] for e in evs)
    padded = [pad_events(e, width) for e in evs]
    return Events(*[np.concatenate([getattr(e, f) for e in padded], axis=0) for f in Events._fields])


# ------------------------------------------------------------------------------------------------
# forward-mode Jacobian
# ------------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class Slot:
    """A free parameter: SimParams field and pool index (fitting/params.py:38-63, plain values)."""
    field: str
    index: int | None
    scale: float = 1.0


def write_params(p: Params, x_phys, slots) -> Params:
    """Physical values written into the named fields (fitting/params.py:100-112)."""
    upd = {}
    for v, s in zip(x_phys, slots):
        if s.index is None:
            upd[s.field] = np.asarray(v)
        else:
            cur = np.array(upd.get(s.field, getattr(p, s.field)), dtype=np.result_type(getattr(p, s.field), v))
            cur[s.index] = v
            upd[s.field] = cur
    return p._replace(**upd)


_CSTEP = 1e-30


def _dsystem(p: Params, slot: Slot, amp, phase, freq):
    """(dA, dC) with respect to one field value, by a complex step through bmc_system."""
    base = getattr(p, slot.field)
    pert = np.array(base, np.complex128)
    if slot.index is None:
        pert = pert + 1j * _CSTEP
    else:
        pert[slot.index] += 1j * _CSTEP
    q = p._replace(**{slot.field: pert})
    A, C = bmc_system(q, amp, phase, freq)
    return np.imag(A) / _CSTEP, np.imag(C) / _CSTEP


def chain_with_tangents(p: Params, ev_row: Events, M0, slots, dM0=None, reset_after_adc=True):
    """last_M and its derivatives with respect to each slot's field value: (N,), (P, N)."""
    nc = n_cest_of(p)
    P = len(slots)
    M = np.asarray(M0, np.float64).copy()
    dM = np.zeros((P, M.size)) if dM0 is None else np.asarray(dM0, np.float64).copy()
    M_init, dM_init = M.copy(), dM.copy()
    last, dlast = M.copy(), dM.copy()
    for j in range(len(ev_row.dt)):
        t = int(ev_row.type[j])
        dt = float(ev_row.dt[j])
        if dt > 1e-9:
            a, ph, fr = float(ev_row.rf_amp[j]), float(ev_row.rf_phase[j]), float(ev_row.rf_freq[j])
            A, C = bmc_system(p, a, ph, fr)
            X = augmented(A, C, dt)
            v = np.append(M, 1.0)
            E = sla.expm(X)
            new_dM = np.empty_like(dM)
            for q, s in enumerate(slots):
                dA, dC = _dsystem(p, s, a, ph, fr)
                _, L = sla.expm_frechet(X, augmented(dA, dC, dt))
                new_dM[q] = (E @ np.append(dM[q], 0.0) + L @ v)[:-1]
            M, dM = (E @ v)[:-1], new_dM
        if t == GRADIENT or t == SPOILER:
            M = _spoil(M, nc)
            dM = np.stack([_spoil(d, nc) for d in dM]) if P else dM
        last, dlast = M, dM
        if t == ADC and reset_after_adc:
            M, dM = M_init.copy(), dM_init.copy()
    return last, dlast


def spectrum_jacobian(p: Params, ev: Events, M0, slots, mz=None):
    """(Z, J): water Mz at every offset and dZ/d(field value) for each slot, (n_off,), (n_off, P)."""
    nc = n_cest_of(p)
    mz = mz_loc(nc) if mz is None else mz
    Z, J = [], []
    for i in range(ev.dt.shape[0]):
        m, dm = chain_with_tangents(p, event_row(ev, i), M0, slots)
        Z.append(m[mz])
        J.append(dm[:, mz])
    return np.array(Z), np.array(J).reshape(len(Z), len(slots))


# ------------------------------------------------------------------------------------------------
# Levenberg-Marquardt (fitting/lm.py:20-67) and the joint trial step (fitting/joint.py:149-162)
# ------------------------------------------------------------------------------------------------
def levenberg_marquardt(resid_jac, x0, lo, hi, n_iter=40, lam0=1e-2, free=None, trajectory=False):
    """Damped Gauss-Newton with fixed iterations. `resid_jac(x)` -> (r, J) at x (scaled units)."""
    x = np.asarray(x0, np.float64).copy()
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    P = x.size
    lam = float(lam0)
    X_tr, C_tr = [], []
    for _ in range(n_iter):
        r, J = resid_jac(x)
        c = float(r @ r)
        if free is not None:
            J = J * free
        g = J.T @ r
        H = J.T @ J
        A = H + lam * (np.diag(np.diag(H)) + 1e-9 * np.eye(P))
        if free is not None:
            A = A + np.diag(1.0 - free)
        delta = np.linalg.solve(A, -g)
        xn = np.clip(x + delta, lo, hi)
        rn, _ = resid_jac(xn, need_jac=False) if _accepts_need_jac(resid_jac) else resid_jac(xn)
        cn = float(rn @ rn)
        better = cn < c
        x = xn if better else x
        lam = lam * 0.5 if better else lam * 3.0
        X_tr.append(x.copy())
        C_tr.append(cn if better else c)
    if trajectory:
        return x, np.array(X_tr), np.array(C_tr)
    return x


def _accepts_need_jac(fn):
    import inspect
    try:
        return "need_jac" in inspect.signature(fn).parameters
    except (TypeError, ValueError):
        return False


def lm_trial(x, lam, J, r, lo, hi, active_bounds=False):
    """The clipped trial point of one damped step; `active_bounds` holds railed values whose step
    points out of the box (fitting/joint.py:149-162)."""
    g, H = J.T @ r, J.T @ J
    P = x.size
    if active_bounds:
        keep = np.where(((x <= lo) & (g > 0)) | ((x >= hi) & (g < 0)), 0.0, 1.0)
        H = H * keep[:, None] * keep[None, :] + np.diag(1.0 - keep)
        g = g * keep
    return np.clip(x + np.linalg.solve(H + lam * (np.diag(np.diag(H)) + 1e-9 * np.eye(P)), -g), lo, hi)


def fit_voxel(p: Params, ev: Events, M0, slots, z_meas, x0_phys, lo_phys, hi_phys, n_iter=30,
              lam0=1e-2, mz=None, trajectory=False):
    """`fit` for one sample: LM in scaled units on r = Z(x) - z_meas (fitting/independent.py:100-129)."""
    sc = np.array([s.scale for s in slots], np.float64)
    z_meas = np.asarray(z_meas, np.float64)

    def rj(xs, need_jac=True):
        q = write_params(p, xs * sc, slots)
        if need_jac:
            Z, J = spectrum_jacobian(q, ev, M0, slots, mz)
            return Z - z_meas, J * sc[None, :]
        nc = n_cest_of(q)
        Z = simulate_spectrum(q, ev, M0)[:, mz_loc(nc) if mz is None else mz]
        return Z - z_meas, None

    out = levenberg_marquardt(rj, np.asarray(x0_phys) / sc, np.asarray(lo_phys) / sc,
                              np.asarray(hi_phys) / sc, n_iter=n_iter, lam0=lam0, trajectory=trajectory)
    if trajectory:
        x, X, C = out
        return x * sc, X * sc[None, :], C
    return out * sc


# ------------------------------------------------------------------------------------------------
# the C twin (oracle/bmc_oracle.c): same algorithm family, compiled, OpenMP over chains
# ------------------------------------------------------------------------------------------------
def c_oracle():
    """ctypes handle of oracle/_build/liboracle.so (built on demand with gcc)."""
    import ctypes as C
    from pathlib import Path
    here = Path(__file__).resolve().parent
    so = here / "_build" / "liboracle.so"
    if not so.exists():
        import subprocess, sys
        subprocess.run([sys.executable, str(here / "build.py")], check=True)
    L = C.CDLL(str(so))
    d, i = C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.oracle_simulate.argtypes = [C.c_int] * 4 + [d, i, d, d, d, d, d, C.c_int, d, C.c_int]
    L.oracle_simulate.restype = C.c_int
    L.oracle_threads.restype = C.c_int
    return L


def c_simulate_z(params_soa, ev: Events, m0, n_cest, mz, threads=0):
    """Z[v][o] from the C oracle. params_soa: [13 + 5 n_cest][n_vox] float64 (the C ABI layout)."""
    import ctypes as C
    L = c_oracle()
    P = np.ascontiguousarray(params_soa, np.float64)
    nv = P.shape[1]
    n_off, n_ev = np.shape(ev.dt)
    t = np.ascontiguousarray(ev.type, np.int32)
    arr = [np.ascontiguousarray(getattr(ev, f), np.float64) for f in ("dt", "rf_amp", "rf_phase", "rf_freq")]
    m = np.ascontiguousarray(np.broadcast_to(np.asarray(m0, np.float64), (nv, state_size(n_cest))))
    out = np.empty((nv, n_off))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    L.oracle_simulate(nv, n_off, n_ev, n_cest, dp(P), t.ctypes.data_as(C.POINTER(C.c_int)), *[dp(a) for a in arr],
                      dp(m), int(mz), dp(out), int(threads))
    return out


# ------------------------------------------------------------------------------------------------
# the damped joint step with one shared value (fitting/joint.py:149-162), dense and by Schur complement
# ------------------------------------------------------------------------------------------------
def joint_step_dense(H, g, free, lam, S):
    """Dense solve of (H + lam (diag H + 1e-9 I)) d = -g over every voxel's local values and (S = 1) one
    value shared by all, assembled from per-voxel blocks H [n][P][P], g [n][P] (shared last), held
    local values (free 0) with identity rows. Returns (d_local [n][PL], d_shared)."""
    H, g, free = np.asarray(H, float), np.asarray(g, float), np.asarray(free, float)
    n, P = g.shape
    PL = P - S
    dim = n * PL + S
    A, b = np.zeros((dim, dim)), np.zeros(dim)
    f = np.concatenate([free.ravel(), np.ones(S)])
    for i in range(n):
        idx = list(range(i * PL, (i + 1) * PL)) + ([n * PL] if S else [])
        A[np.ix_(idx, idx)] += H[i]
        b[idx] += g[i]
    A = A * f[:, None] * f[None, :]
    b = b * f
    A = A + lam * (np.diag(np.diag(A)) + 1e-9 * np.eye(dim)) + np.diag(1.0 - f)
    d = np.linalg.solve(A, -b)
    return d[:n * PL].reshape(n, PL), (d[-1] if S else 0.0)


def schur_partial(H, g, free, lam, S):
    """One shard's part of the Schur-complement step: per voxel Y = A^-1 h_ps, w = A^-1 g_p, and the four
    sums (h_ss, h_ps^T Y, h_ps^T w, g_s) over the shard's voxels."""
    H, g, free = np.asarray(H, float), np.asarray(g, float), np.asarray(free, float)
    n, P = g.shape
    PL = P - S
    Y, w, sums = np.zeros((n, PL)), np.zeros((n, PL)), np.zeros(4)
    for i in range(n):
        fr = free[i]
        A = H[i, :PL, :PL] * np.outer(fr, fr) + np.diag(fr * lam * (np.diag(H[i, :PL, :PL]) + 1e-9) + (1 - fr))
        hps = fr * H[i, :PL, PL] if S else np.zeros(PL)
        Y[i] = np.linalg.solve(A, hps)
        w[i] = np.linalg.solve(A, fr * g[i, :PL])
        if S:
            sums += [H[i, PL, PL], hps @ Y[i], hps @ w[i], g[i, PL]]
    return Y, w, sums


def schur_back(Y, w, sums, lam, S):
    """The shared step from the sums of every shard, then each voxel's: (d_local, d_shared)."""
    hss, sy, tw, gs = sums
    ds = -(gs - tw) / (hss + lam * (hss + 1e-9) - sy) if S else 0.0
    return -(w + Y * ds), ds
