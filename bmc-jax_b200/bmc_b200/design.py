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

__all__ = ["crlb", "CRLB", "fisher_information", "model_of", "jacobian", "optimize_design", "DesignResult"]


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


def optimize_design(build: Callable, spec: FitSpec, d0, lo, hi, sigma: float, truths,
                    targets: Optional[Sequence[str]] = None, n_steps: int = 200, lr: float = 0.05,
                    callback: Optional[Callable] = None, rel_step: float = 1e-4) -> DesignResult:
    """Lower the Cramer-Rao bound of the target parameters by changing the design (design/optimize.py:43-113).

    `build(d) -> Experiment` (one sample) from a design vector d, here with NumPy operations. The cost,
    its parametrisation d = lo + (hi - lo) sigmoid(u) and the Adam steps on u are the reference's. The
    reference differentiates the cost with respect to d by automatic differentiation through the bound;
    here the Jacobian inside the bound is the exact forward-mode tangent of the GPU kernel and the outer
    derivative is a central difference in each setting with step rel_step * (hi - lo): 2 len(d) + 1
    bound evaluations (one launch each, every truth in it) per step, float64 throughout."""
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
        c = cost_of(d)
        gd = np.empty_like(d)
        for i in range(d.size):
            e = np.zeros_like(d)
            e[i] = h[i]
            gd[i] = (cost_of(d + e) - cost_of(d - e)) / (2.0 * h[i])
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
