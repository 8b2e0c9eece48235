"""The Cramer-Rao lower bound of a protocol (BMC-JAX design/crlb.py:38-120) on the GPU tangents.

F = J^T J / sigma^2 with J = dZ/dx from the forward-mode kernel (float64); the inverse, the standard
deviations and the correlations are formed on the host in float64, as the reference does.
"""
from dataclasses import dataclass

import numpy as np

from . import _lib
from .fitting import FitSpec, field_row, write_params
from .simulation import (SimEvent, n_cest_of, n_samples, pack_params, state_size, DeviceEvents, problem,
                         _device)

__all__ = ["crlb", "CRLB", "fisher_information", "model_of", "jacobian"]


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
    names: tuple
    x: np.ndarray
    sd: np.ndarray
    corr: np.ndarray
    fisher: np.ndarray
    jacobian: np.ndarray

    @property
    def rel_sd(self) -> np.ndarray:
        return self.sd / np.abs(self.x)

    def __getitem__(self, name: str) -> float:
        return float(self.sd[self.names.index(name)])

    def summary(self) -> str:
        rows = [f"{'parameter':>10} {'value':>12} {'CRLB (SD)':>12} {'relative':>9}"]
        for n, x, s, r in zip(self.names, self.x, self.sd, self.rel_sd):
            rows.append(f"{n:>10} {x:>12.6g} {s:>12.4g} {100 * r:>8.2f}%")
        return "\n".join(rows)


def crlb(experiment, spec: FitSpec, sigma, x=None) -> CRLB:
    """The Cramer-Rao lower bound of `spec`'s parameters for one sample (crlb.py:88-120)."""
    x = np.asarray(spec.x0_phys if x is None else x, float)
    F, J = fisher_information(experiment, spec, x, sigma)
    F = np.asarray(F, np.float64)
    cov = np.linalg.inv(F)
    sd = np.sqrt(np.clip(np.diag(cov), 0.0, None))
    corr = cov / np.outer(sd, sd)
    return CRLB(tuple(s.name for s in spec.slots), x, sd, corr, F, np.asarray(J))
