"""The Cramer-Rao lower bound of a protocol (BMC-JAX design/crlb.py:38-120) on the GPU tangents.

F = J^T J / sigma^2 with J = dZ/dx from the forward-mode kernel (float64); the inverse, the standard
deviations and the correlations are formed on the host in float64, as the reference does.
"""
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib
from .fitting import FitSpec, field_row, write_params
from .simulation import (SimEvent, n_cest_of, n_samples, pack_params, state_size, DeviceEvents, problem,
                         _device)

__all__ = ["crlb", "CRLB", "fisher_information", "model_of", "jacobian", "optimize_design", "DesignResult",
           "design_cost", "design_cost_and_gradient", "design_jacobians"]


def _check(experiment, spec: FitSpec):
    if n_samples(experiment.params) is not None:
        raise ValueError("the bound is computed for one sample: give an Experiment whose params carry one sample")
    if not spec.independent:
        raise ValueError("the bound supports plain values per sample (FreeParam scope='sample', mode='value', no "
                         "samples=, no m_start or b0_spread)")


def jacobian(experiment, spec: FitSpec, x_phys):
    """(Z, J): water Mz at every offset and dZ/dx (physical units) at x_phys, from the GPU tangents."""
    torch = _lib.torch_cuda()
    base = experiment.params
    nc = n_cest_of(base)
    x_phys = np.asarray(x_phys, np.float64)
    p = write_params(base, x_phys / spec.scales, spec)
    dev_ev = DeviceEvents(experiment.events)
    pdev = _device(pack_params(p, 1))
    mdev = _device(np.asarray(experiment.m0, np.float64).reshape(1, state_size(nc)))
    P = spec.n
    z = torch.empty((1, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
    jz = torch.empty((P, 1, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
    tg = _lib.Tangents()
    tg.n_tangents = P
    for i, s in enumerate(spec.slots):
        tg.field_row[i] = field_row(s.field, s.index, nc)
    seed = _device(np.ones((P, 1)))
    tg.d_seed = seed.data_ptr()
    tg.d_dm0 = None
    pr = problem(1, dev_ev.n_offsets, dev_ev.n_events, nc, int(experiment.mz_loc), _lib.F64)
    _lib.check(_lib.lib().bmc_simulate_jvp(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev), None, tg,
                                           _lib.ptr(z), _lib.ptr(jz), _lib.stream_handle()))
    return z.cpu().numpy()[0], jz.cpu().numpy()[:, 0, :].T


def model_of(experiment, spec: FitSpec):
    """x (physical) -> Z, the model `fit` inverts (crlb.py:38-47)."""
    _check(experiment, spec)
    return lambda x: jacobian(experiment, spec, x)[0]


def fisher_information(experiment, spec: FitSpec, x, sigma):
    """(F, J): F = J^T J / sigma^2 at x (physical units) (crlb.py:50-58)."""
    _check(experiment, spec)
    _, J = jacobian(experiment, spec, x)
    return J.T @ J / sigma ** 2, J


@dataclass(frozen=True)
class CRLB:
    """The bound at the values x (the fields of BMC-JAX design/crlb.py:61-85): per parameter the smallest
    standard deviation an unbiased estimate can have (sd), the correlations, the Fisher matrix and the
    Jacobian it came from."""
    names: tuple
    x: np.ndarray
    sd: np.ndarray
    corr: np.ndarray
    fisher: np.ndarray
    jacobian: np.ndarray

    @property
    def rel_sd(self) -> np.ndarray:
        """sd / |x|."""
        return np.asarray(self.sd) / np.abs(np.asarray(self.x))

    def __getitem__(self, name: str) -> float:
        """The bound (sd) of one parameter by its name (ValueError for a name not in the bound)."""
        bound = dict(zip(self.names, np.asarray(self.sd)))
        if name not in bound:
            raise ValueError(f"{name!r} is not one of {self.names}")
        return float(bound[name])

    def summary(self) -> str:
        """One line per parameter: value, bound and the bound relative to the value."""
        return "\n".join(f"{n}: {x:.6g} +- {s:.4g} (CRLB, {100 * r:.2f}% of the value)"
                         for n, x, s, r in zip(self.names, self.x, self.sd, self.rel_sd))


def crlb(experiment, spec: FitSpec, sigma, x=None) -> CRLB:
    """The Cramer-Rao lower bound of `spec`'s parameters for one sample (crlb.py:88-120)."""
    x = np.asarray(spec.x0_phys if x is None else x, float)
    F, J = fisher_information(experiment, spec, x, sigma)
    F = np.asarray(F, np.float64)
    cov = np.linalg.inv(F)
    sd = np.sqrt(np.clip(np.diag(cov), 0.0, None))
    corr = cov / np.outer(sd, sd)
    return CRLB(tuple(s.name for s in spec.slots), x, sd, corr, F, np.asarray(J))


# ------------------------------------------------------------------------------------------------
# protocol optimisation (design/optimize.py:43-113)
# ------------------------------------------------------------------------------------------------
def jacobians(experiment, spec: FitSpec, X_phys):
    """dZ/dx (physical units) of one Experiment at every row of X_phys: (n, n_offsets, P), one launch."""
    from .simulation import tile_params
    torch = _lib.torch_cuda()
    _check(experiment, spec)
    X = np.atleast_2d(np.asarray(X_phys, np.float64))
    n = X.shape[0]
    nc = n_cest_of(experiment.params)
    p = write_params(tile_params(experiment.params, n), X / spec.scales, spec)
    dev_ev = DeviceEvents(experiment.events)
    pdev = _device(pack_params(p, n))
    mdev = _device(np.broadcast_to(np.asarray(experiment.m0, np.float64).reshape(1, -1), (n, state_size(nc))))
    P = spec.n
    z = torch.empty((n, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
    jz = torch.empty((P, n, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
    tg = _lib.Tangents()
    tg.n_tangents = P
    for i, sl in enumerate(spec.slots):
        tg.field_row[i] = field_row(sl.field, sl.index, nc)
    seed = _device(np.ones((P, n)))
    tg.d_seed = seed.data_ptr()
    tg.d_dm0 = None
    pr = problem(n, dev_ev.n_offsets, dev_ev.n_events, nc, int(experiment.mz_loc), _lib.F64)
    _lib.check(_lib.lib().bmc_simulate_jvp(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev), None, tg,
                                           _lib.ptr(z), _lib.ptr(jz), _lib.stream_handle()))
    return jz.cpu().numpy().transpose(1, 2, 0)


@dataclass(frozen=True)
class DesignResult:
    """The optimised design and how much it lowered the bound (design/optimize.py:29-38)."""
    design: np.ndarray
    start: np.ndarray
    cost: np.ndarray
    targets: tuple
    truths: np.ndarray
    rel_sd_start: np.ndarray
    rel_sd_end: np.ndarray


def design_cost(build: Callable, spec: FitSpec, d, sigma: float, truths, targets: Sequence[str]) -> float:
    """Mean over the truths of sum over the targets of (SD_j / x_j)^2, the bound from the GPU tangents."""
    names = [sl.name for sl in spec.slots]
    idx = np.array([names.index(t) for t in targets])
    truths = np.atleast_2d(np.asarray(truths, np.float64))
    J = jacobians(build(np.asarray(d, np.float64)), spec, truths)
    total = 0.0
    for x, Jx in zip(truths, J):
        var = np.diag(np.linalg.inv(Jx.T @ Jx / sigma ** 2))[idx]
        total += float(np.sum(var / x[idx] ** 2))
    return total / truths.shape[0]


_EV_FIELDS = ("dt", "rf_amp", "rf_phase", "rf_freq")


def _build_direction(build: Callable, d, i: int, h: float, ref):
    """The derivative of build(d) with respect to setting i: (events, packed params [n_fields], m0) per unit
    of d_i, by the five-point stencil (-f(+2h) + 8 f(+h) - 8 f(-h) + f(-2h)) / 12h of the host build,
    which is exact to rounding wherever build is affine in d_i (amplitudes, durations and offsets scaled
    or shifted by a setting), O(h^4) otherwise. Everything after the build is differentiated exactly."""
    pts = {}
    for k in (-2, -1, 1, 2):
        dd = np.array(d, np.float64, copy=True)
        dd[i] += k * h
        ex = build(dd)
        ev = ex.events
        if np.shape(ev.dt) != np.shape(ref.events.dt) or not np.array_equal(np.asarray(ev.type),
                                                                          np.asarray(ref.events.type)):
            raise ValueError(f"build(d) must keep the event table's shape and event types as setting {i} moves")
        if int(ex.mz_loc) != int(ref.mz_loc) or n_cest_of(ex.params) != n_cest_of(ref.params):
            raise ValueError(f"build(d) must keep the pools and mz_loc as setting {i} moves")
        pts[k] = ([np.asarray(getattr(ev, f), np.float64) for f in _EV_FIELDS], pack_params(ex.params, 1)[:, 0],
                  np.asarray(ex.m0, np.float64).reshape(-1))
    # the differences first: an entry the setting does not move gets exactly zero
    st = lambda a2, a1, m1, m2: (8.0 * (a1 - m1) - (a2 - m2)) / (12.0 * h)
    ev = [st(pts[2][0][j], pts[1][0][j], pts[-1][0][j], pts[-2][0][j]) for j in range(len(_EV_FIELDS))]
    return ev, st(pts[2][1], pts[1][1], pts[-1][1], pts[-2][1]), st(pts[2][2], pts[1][2], pts[-1][2], pts[-2][2])


def design_jacobians(build: Callable, spec: FitSpec, d, X_phys, steps):
    """(J, dJ) at design d: J = dZ/dx (physical units) at every row of X_phys, (n, n_offsets, P), and dJ its
    derivative with respect to every setting of d, (len(d), n, n_offsets, P), from the second-order kernel
    (bmc_simulate_design_jvp: forward mode over forward mode through the whole simulation, one launch per
    tangent and setting). `steps[i]` is the stencil step that differentiates the host build in d_i
    (_build_direction). The fitted fields are set by x, so the design moves only the others."""
    from .simulation import tile_params
    torch = _lib.torch_cuda()
    d = np.asarray(d, np.float64)
    exp = build(d)
    _check(exp, spec)
    X = np.atleast_2d(np.asarray(X_phys, np.float64))
    n = X.shape[0]
    nc = n_cest_of(exp.params)
    N = state_size(nc)
    P = spec.n
    rows = [field_row(sl.field, sl.index, nc) for sl in spec.slots]
    p = write_params(tile_params(exp.params, n), X / spec.scales, spec)
    dev_ev = DeviceEvents(exp.events)
    n_off = dev_ev.n_offsets
    pdev = _device(pack_params(p, n))
    mdev = _device(np.broadcast_to(np.asarray(exp.m0, np.float64).reshape(1, -1), (n, N)))
    tg = _lib.Tangents()
    tg.n_tangents = P
    for t, r in enumerate(rows):
        tg.field_row[t] = r
    seed = _device(np.ones((P, n)))
    tg.d_seed = seed.data_ptr()
    tg.d_dm0 = None
    pr = problem(n, n_off, dev_ev.n_events, nc, int(exp.mz_loc), _lib.F64)
    f64 = dict(dtype=torch.float64, device="cuda")
    z, jz = torch.empty((n, n_off), **f64), torch.empty((P, n, n_off), **f64)
    dz, djz = torch.empty((n, n_off), **f64), torch.empty((P, n, n_off), **f64)
    J, dJ = None, np.empty((d.size, n, n_off, P))
    for i in range(d.size):
        ev_d, p_d, m_d = _build_direction(build, d, i, float(steps[i]), exp)
        p_d = np.repeat(p_d.reshape(-1, 1), n, axis=1)
        p_d[rows] = 0.0
        evd = [_device(a) for a in ev_d]
        ev_struct = _lib.Events(0, evd[0].data_ptr(), evd[1].data_ptr(), evd[2].data_ptr(), evd[3].data_ptr(), 0)
        pd_dev = _device(p_d)
        md_dev = _device(np.broadcast_to(m_d.reshape(1, -1), (n, N)))
        _lib.check(_lib.lib().bmc_simulate_design_jvp(pr, _lib.ptr(pdev), dev_ev.struct, _lib.ptr(mdev),
                                                      _lib.ptr(pd_dev), ev_struct, _lib.ptr(md_dev), tg, _lib.ptr(z),
                                                      _lib.ptr(jz), _lib.ptr(dz), _lib.ptr(djz),
                                                      _lib.stream_handle()))
        if J is None:
            J = jz.cpu().numpy().transpose(1, 2, 0)
        dJ[i] = djz.cpu().numpy().transpose(1, 2, 0)
    return J, dJ


def design_cost_and_gradient(build: Callable, spec: FitSpec, d, sigma: float, truths, targets: Sequence[str],
                             steps):
    """(cost, d cost / d d): the cost of design_cost and its exact gradient. With F = J^T J / sigma^2 and
    var = diag(F^-1), a setting's dJ gives dF = (dJ^T J + J^T dJ) / sigma^2 and d var = -diag(F^-1 dF F^-1)."""
    names = [sl.name for sl in spec.slots]
    idx = np.array([names.index(t) for t in targets])
    truths = np.atleast_2d(np.asarray(truths, np.float64))
    J, dJ = design_jacobians(build, spec, d, truths, steps)
    cost, grad = 0.0, np.zeros(dJ.shape[0])
    for k, x in enumerate(truths):
        Jx = J[k]
        Fi = np.linalg.inv(Jx.T @ Jx / sigma ** 2)
        w = 1.0 / x[idx] ** 2
        cost += float(np.sum(np.diag(Fi)[idx] * w))
        for i in range(dJ.shape[0]):
            dF = (dJ[i, k].T @ Jx + Jx.T @ dJ[i, k]) / sigma ** 2
            grad[i] -= float(np.sum(np.diag(Fi @ dF @ Fi)[idx] * w))
    return cost / truths.shape[0], grad / truths.shape[0]


def optimize_design(build: Callable, spec: FitSpec, d0, lo, hi, sigma: float, truths,
                    targets: Optional[Sequence[str]] = None, n_steps: int = 200, lr: float = 0.05,
                    callback: Optional[Callable] = None, rel_step: float = 1e-3) -> DesignResult:
    """Lower the Cramer-Rao bound of the target parameters by changing the design (design/optimize.py:43-113).

    `build(d) -> Experiment` (one sample) from a design vector d, here with NumPy operations. The cost,
    its parametrisation d = lo + (hi - lo) sigmoid(u) and the Adam steps on u are the reference's. The
    reference differentiates the cost with respect to d by automatic differentiation through the bound;
    here the gradient is exact from the simulation on: the second-order kernel (bmc_simulate_design_jvp)
    carries each setting's direction and every parameter tangent through the whole simulation at once
    (design_cost_and_gradient). NumPy cannot be traced, so the build itself is differentiated by a
    five-point stencil with step rel_step * (hi - lo) (exact to rounding for builds affine in each
    setting, such as scaled amplitudes). float64 throughout."""
    names = [sl.name for sl in spec.slots]
    targets = tuple(names if targets is None else targets)
    unknown = [t for t in targets if t not in names]
    if unknown:
        raise ValueError(f"targets {unknown} are not parameters of the spec {names}")
    truths = np.atleast_2d(np.asarray(truths, float))
    d0, lo, hi = (np.asarray(a, float) for a in (d0, lo, hi))
    if not (d0.shape == lo.shape == hi.shape) or np.any(d0 <= lo) or np.any(d0 >= hi):
        raise ValueError("d0, lo and hi need the same shape, with lo < d0 < hi")
    sig = lambda u: 1.0 / (1.0 + np.exp(-u))
    to_d = lambda u: lo + (hi - lo) * sig(u)
    cost_of = lambda d: design_cost(build, spec, d, sigma, truths, targets)
    p0 = (d0 - lo) / (hi - lo)
    u = np.log(p0 / (1.0 - p0))
    h = rel_step * (hi - lo)
    m, v, b1, b2, eps = np.zeros_like(u), np.zeros_like(u), 0.9, 0.999, 1e-8
    history = []
    for step in range(int(n_steps)):
        d = to_d(u)
        c, gd = design_cost_and_gradient(build, spec, d, sigma, truths, targets, h)
        g = gd * (hi - lo) * sig(u) * (1.0 - sig(u))
        if not (np.isfinite(c) and np.all(np.isfinite(g))):
            raise FloatingPointError(f"cost or gradient not finite at step {step}; try a smaller lr")
        history.append(c)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g ** 2
        u = u - lr * (m / (1 - b1 ** (step + 1))) / (np.sqrt(v / (1 - b2 ** (step + 1))) + eps)
        if callback is not None:
            callback(step, c, to_d(u))
    design = to_d(u)
    history.append(cost_of(design))

    def rel(dd):
        exp = build(np.asarray(dd, float))
        return np.array([[crlb(exp, spec, sigma, x).rel_sd[names.index(t)] for t in targets] for x in truths])
    return DesignResult(design, d0, np.asarray(history), targets, truths, rel(d0), rel(design))
