"""Learned warm start for the Levenberg-Marquardt fit (an addition of this library; BMC-JAX has none).

A multilayer perceptron maps a measured saturation ladder (the Z values of a stacked Experiment) to
starting values of the free parameters; the LM fit (`fitting.fit`, every iteration on the GPU) then
starts from there instead of from the FitSpec's fixed x0 and needs fewer iterations. The plain fit
from the fixed x0 stays the fallback and the judge: a voxel whose warm-started fit ends with an rms
residual above `fallback_rms` is refitted plainly, and the better of the two fits is kept.

The network is trained on spectra that the simulator itself generates (parameters drawn uniformly
from the training ranges, Gaussian noise added), with the library's own kernels: bf16 tcgen05 GEMMs
with fp32 accumulation for the forward and backward passes and an Adam step on fp32 master weights
(csrc/bmc_mlp.cu, entry points bmc_mlp_*). There is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib

__all__ = ["MLP", "LadderWarmStart", "WarmFitResult"]


def _rup(x, m):
    return (x + m - 1) // m * m


class MLP:
    """x (n_in) -> n_hidden_layers x [affine, GELU] of width n_hidden -> affine -> y (n_out), on the GPU.

    Parameters live on the device as float32 master weights (`params`, layout of bmc_mlp_* in
    include/bmc_b200.h) with a bf16 shadow (W and W^T per layer) that the tensor cores read. Inputs
    are normalised per feature by (x - in_shift) * in_scale inside the input kernel."""

    def __init__(self, n_in: int, n_out: int, n_hidden: int = 256, n_hidden_layers: int = 3, seed: int = 0):
        torch = _lib.torch_cuda()
        self.shape = _lib.MlpShape(int(n_in), int(n_hidden), int(n_hidden_layers), int(n_out))
        self.n_in, self.n_out = int(n_in), int(n_out)
        L = _lib.lib()
        n_p, sh_b, _ = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.check(L.bmc_mlp_sizes(C.byref(self.shape), 1, C.byref(n_p), C.byref(sh_b), None))
        self.n_params = int(n_p.value)
        self.params = torch.as_tensor(self.init_params(n_in, n_hidden, n_hidden_layers, n_out, seed)).to("cuda")
        if self.params.numel() != self.n_params:
            raise RuntimeError("parameter layout disagrees with the library")
        self.shadow = torch.zeros(int(sh_b.value), dtype=torch.uint8, device="cuda")
        self.grad = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.in_shift = torch.zeros(n_in, dtype=torch.float32, device="cuda")
        self.in_scale = torch.ones(n_in, dtype=torch.float32, device="cuda")
        self.step = 0
        self._work: Dict[int, object] = {}
        self.sync()

    # -- layout ---------------------------------------------------------------------------------
    @staticmethod
    def layout(n_in, n_hidden, n_layers, n_out) -> List[Tuple[int, int, int, int]]:
        """(off_w, off_b, rows, cols) per layer: hidden layers then the output layer, padded to 64."""
        in_pad, out_pad = _rup(n_in, 64), _rup(n_out, 64)
        dims = [(n_hidden, in_pad)] + [(n_hidden, n_hidden)] * (n_layers - 1) + [(out_pad, n_hidden)]
        out, off = [], 0
        for r, c in dims:
            out.append((off, off + r * c, r, c))
            off += r * c + r
        return out

    @classmethod
    def init_params(cls, n_in, n_hidden, n_layers, n_out, seed=0) -> np.ndarray:
        """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) on the real weights and biases; zero padding."""
        lay = cls.layout(n_in, n_hidden, n_layers, n_out)
        rng = np.random.default_rng(seed)
        p = np.zeros(lay[-1][1] + lay[-1][2], np.float32)
        fan_in = [n_in] + [n_hidden] * n_layers
        real_out = [n_hidden] * n_layers + [n_out]
        for (ow, ob, r, c), fi, ro in zip(lay, fan_in, real_out):
            bound = 1.0 / np.sqrt(fi)
            W = np.zeros((r, c), np.float32)
            W[:ro, :fi] = rng.uniform(-bound, bound, (ro, fi))
            p[ow:ob] = W.ravel()
            p[ob:ob + ro] = rng.uniform(-bound, bound, ro)
        return p

    # -- device plumbing ------------------------------------------------------------------------
    def sync(self):
        """Rebuild the bf16 shadow from the float32 master weights."""
        _lib.check(_lib.lib().bmc_mlp_sync(C.byref(self.shape), _lib.ptr(self.params), _lib.ptr(self.shadow),
                                           _lib.stream_handle()))

    def work(self, batch: int):
        w = self._work.get(batch)
        if w is None:
            torch = _lib.torch_cuda()
            wb = C.c_int64()
            _lib.check(_lib.lib().bmc_mlp_sizes(C.byref(self.shape), int(batch), None, None, C.byref(wb)))
            w = torch.zeros(int(wb.value), dtype=torch.uint8, device="cuda")
            self._work[batch] = w
        return w

    def status(self, batch: int) -> int:
        """The status word of a work buffer (bit 0: a GEMM gave up waiting on the tensor core)."""
        w = self.work(batch)
        return int(w[:4].view(_lib.torch_cuda().int32)[0].item())

    def set_input_normalisation(self, shift, scale):
        torch = _lib.torch_cuda()
        self.in_shift = torch.as_tensor(np.asarray(shift, np.float32)).to("cuda")
        self.in_scale = torch.as_tensor(np.asarray(scale, np.float32)).to("cuda")

    # -- forward, backward, Adam ----------------------------------------------------------------
    def forward(self, x, keep: bool = False):
        """y [batch][n_out] (float32, device) for x [batch][n_in] (float32, device)."""
        torch = _lib.torch_cuda()
        x = x.contiguous()
        if x.dtype != torch.float32 or x.dim() != 2 or x.shape[1] != self.n_in:
            raise ValueError(f"x must be float32 [batch][{self.n_in}] on the device")
        b = int(x.shape[0])
        y = torch.empty((b, self.n_out), dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().bmc_mlp_forward(C.byref(self.shape), _lib.ptr(self.params), _lib.ptr(self.shadow),
                                              _lib.ptr(x), _lib.ptr(self.in_shift), _lib.ptr(self.in_scale), b,
                                              _lib.ptr(y), _lib.ptr(self.work(b)), 1 if keep else 0,
                                              _lib.stream_handle()))
        return y

    def backward(self, target, loss=None):
        """Gradients (into self.grad) of the mean squared error of the last forward(keep=True)."""
        target = target.contiguous()
        b = int(target.shape[0])
        _lib.check(_lib.lib().bmc_mlp_backward(C.byref(self.shape), _lib.ptr(self.shadow), _lib.ptr(target), b,
                                               _lib.ptr(self.work(b)), _lib.ptr(self.grad), _lib.ptr(loss),
                                               _lib.stream_handle()))

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        _lib.check(_lib.lib().bmc_mlp_adam_step(C.byref(self.shape), _lib.ptr(self.params), _lib.ptr(self.grad),
                                                _lib.ptr(self.m), _lib.ptr(self.v), _lib.ptr(self.shadow),
                                                self.step, lr, beta1, beta2, eps, _lib.stream_handle()))

    def adam_dev(self, d_step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        """Adam step with the step count in the device int32 `d_step` (advanced by the library)."""
        _lib.check(_lib.lib().bmc_mlp_adam_step_dev(C.byref(self.shape), _lib.ptr(self.params), _lib.ptr(self.grad),
                                                    _lib.ptr(self.m), _lib.ptr(self.v), _lib.ptr(self.shadow),
                                                    _lib.ptr(d_step), lr, beta1, beta2, eps, _lib.stream_handle()))

    def train(self, X, T, epochs: int = 10, batch: int = 4096, lr: float = 1e-3, seed: int = 0,
              graph: bool = True) -> List[float]:
        """Adam on mean squared error over (X, T) (device float32 tensors); returns the mean training
        loss of each epoch. The last partial batch of an epoch is dropped. With `graph`, one training step
        (batch gather, forward, backward, Adam) is captured into a CUDA graph after the first step runs
        eagerly, and replayed for the others; the step count lives on the device for that."""
        torch = _lib.torch_cuda()
        n = int(X.shape[0])
        if n < batch:
            raise ValueError(f"{n} training rows for batch {batch}")
        g = torch.Generator(device="cuda")
        g.manual_seed(int(seed))
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        d_step = torch.tensor([self.step], dtype=torch.int32, device="cuda")
        idx = torch.empty(batch, dtype=torch.int64, device="cuda")

        def one_step():
            xb, tb = X.index_select(0, idx), T.index_select(0, idx)
            self.forward(xb, keep=True)
            self.backward(tb, loss)
            self.adam_dev(d_step, lr)

        hist = []
        steps = n // batch
        captured = None
        try:
            for _ in range(int(epochs)):
                perm = torch.randperm(n, device="cuda", generator=g)
                loss.zero_()
                for s in range(steps):
                    idx.copy_(perm[s * batch:(s + 1) * batch])
                    if captured is not None:
                        captured.replay()
                        continue
                    one_step()
                    if graph:
                        captured = torch.cuda.CUDAGraph()
                        with torch.cuda.graph(captured):
                            one_step()
                hist.append(float(loss.item()) / steps)
        finally:
            del captured
        self.step = int(d_step.item())
        if self.status(batch) != 0:
            raise RuntimeError("a tensor-core GEMM gave up waiting during training (status word set)")
        return hist

    def predict(self, X, batch: int = 65536):
        """y for every row of X (device float32), in batches."""
        torch = _lib.torch_cuda()
        out = [self.forward(X[a:a + batch]) for a in range(0, int(X.shape[0]), batch)]
        return torch.cat(out) if out else torch.empty((0, self.n_out), device="cuda")


@dataclass
class WarmFitResult:
    """What `LadderWarmStart.fit` kept: physical x (n, P), rms (n,), the network's starting values
    x0 (n, P), which voxels were refitted plainly, and wall-clock seconds per stage."""
    x: np.ndarray
    rms: np.ndarray
    x0: np.ndarray
    refit: np.ndarray
    n_iter_warm: int
    n_iter_plain: int
    seconds: Dict[str, float]


class LadderWarmStart:
    """Warm start of `fitting.fit` for one Experiment (one event table, one base parameter set) and a
    FitSpec of per-sample plain values.

    The network reads the Experiment's Z values (all offsets of all stacked rungs) and predicts each
    free parameter normalised to its training range [lo, hi] (`ranges`, by default the FitSpec's
    bounds). `train` draws parameters uniformly from those ranges, simulates the ladder with the
    library's forward model, adds Gaussian noise of `sigma`, and fits the network to the draws."""

    def __init__(self, experiment, spec, ranges: Optional[Sequence[Tuple[float, float]]] = None,
                 sigma: float = 0.005, n_hidden: int = 256, n_hidden_layers: int = 3, seed: int = 0):
        spec.require_independent("LadderWarmStart")
        self.experiment, self.spec, self.sigma = experiment, spec, float(sigma)
        r = ranges if ranges is not None else list(zip(spec.lo_phys, spec.hi_phys))
        self.lo = np.array([a for a, _ in r], np.float64)
        self.hi = np.array([b for _, b in r], np.float64)
        if self.lo.size != spec.n or np.any(self.hi <= self.lo):
            raise ValueError("ranges: one (lo, hi) with lo < hi per free parameter")
        self.n_points = int(np.shape(experiment.events.dt)[0])
        self.mlp = MLP(self.n_points, spec.n, n_hidden, n_hidden_layers, seed)

    # -- the simulator as the data source ------------------------------------------------------
    def simulate(self, X_phys, chunk: int = 131072):
        """Z (float32, device) [n][n_points] of the Experiment with the free parameters set to X_phys. The
        spectra stay on the device: each chunk's float64 Z is rounded into the output there."""
        from .fitting import write_params
        from .simulation import (DeviceEvents, _device, n_cest_of, pack_params, problem, simulate_device,
                                 state_size, tile_params)
        torch = _lib.torch_cuda()
        X_phys = np.asarray(X_phys, np.float64)
        n = X_phys.shape[0]
        out = torch.empty((n, self.n_points), dtype=torch.float32, device="cuda")
        ex = self.experiment
        dev_ev = DeviceEvents(ex.events)
        nc = n_cest_of(ex.params)
        m0 = np.asarray(ex.m0, np.float64).reshape(-1, state_size(nc))
        z = None
        for a in range(0, n, chunk):
            b = min(a + chunk, n)
            p = write_params(tile_params(ex.params, b - a), self.spec.to_scaled(X_phys[a:b]), self.spec)
            pdev = _device(pack_params(p, b - a))
            mdev = _device(np.broadcast_to(m0, (b - a, m0.shape[1])))
            if z is None or z.shape[0] != b - a:
                z = torch.empty((b - a, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
            simulate_device(problem(b - a, dev_ev.n_offsets, dev_ev.n_events, nc, int(ex.mz_loc)), pdev, dev_ev,
                            mdev, z)
            out[a:b] = z.float()
        return out

    def simulate64(self, X_phys, chunk: int = 131072) -> np.ndarray:
        """Z (float64, host) [n][n_points] of the Experiment with the free parameters set to X_phys."""
        from .fitting import write_params
        from .simulation import simulate_z, tile_params
        X_phys = np.asarray(X_phys, np.float64)
        ex = self.experiment
        parts = []
        for a in range(0, X_phys.shape[0], chunk):
            b = min(a + chunk, X_phys.shape[0])
            p = write_params(tile_params(ex.params, b - a), self.spec.to_scaled(X_phys[a:b]), self.spec)
            parts.append(np.asarray(simulate_z(p, ex.events, ex.m0, ex.mz_loc), np.float64))
        return np.concatenate(parts) if parts else np.zeros((0, self.n_points))

    def draw(self, n: int, seed: int) -> np.ndarray:
        """n parameter vectors drawn uniformly from the training ranges (physical units)."""
        rng = np.random.default_rng(seed)
        return self.lo + (self.hi - self.lo) * rng.random((n, self.spec.n))

    def normalise(self, X_phys):
        return (np.asarray(X_phys, np.float64) - self.lo) / (self.hi - self.lo)

    def training_set(self, n: int, seed: int = 0):
        """(Z with noise, normalised targets), both float32 on the device, and the physical draws."""
        torch = _lib.torch_cuda()
        X = self.draw(n, seed)
        Z = self.simulate(X)
        if self.sigma > 0:
            g = torch.Generator(device="cuda")
            g.manual_seed(int(seed) + 1)
            Z += self.sigma * torch.randn(Z.shape, generator=g, device="cuda", dtype=torch.float32)
        T = torch.as_tensor(self.normalise(X).astype(np.float32)).to("cuda")
        return Z, T, X

    def train(self, n_train: int = 2_000_000, epochs: int = 10, batch: int = 4096, lr: float = 1e-3,
              seed: int = 0, data=None) -> List[float]:
        """Train on n_train simulated ladders (or on `data` = (Z, T) already on the device)."""
        Z, T = data if data is not None else self.training_set(n_train, seed)[:2]
        mu = Z.mean(dim=0)
        sd = Z.std(dim=0).clamp_min(1e-6)
        self.mlp.set_input_normalisation(mu.cpu().numpy(), (1.0 / sd).cpu().numpy())
        return self.mlp.train(Z, T, epochs=epochs, batch=batch, lr=lr, seed=seed)

    # -- inference and the warm-started fit ----------------------------------------------------
    def starting_values(self, z) -> np.ndarray:
        """Physical starting values (n, P) for measured Z (n, n_points), clipped into the FitSpec's
        bounds and the training ranges."""
        torch = _lib.torch_cuda()
        zt = z if hasattr(z, "data_ptr") else torch.as_tensor(np.asarray(z, np.float32)).to("cuda")
        y = self.mlp.predict(zt.float()).double().cpu().numpy()
        x = self.lo + (self.hi - self.lo) * np.clip(y, 0.0, 1.0)
        return np.clip(x, np.maximum(self.spec.lo_phys, self.lo), np.minimum(self.spec.hi_phys, self.hi))

    def fit(self, z_meas, n_iter_warm: int = 8, n_iter_plain: int = 30,
            fallback_rms: Optional[float] = None, judge: str = "threshold") -> WarmFitResult:
        """LM from the network's starting values (n_iter_warm iterations), with the plain fit from the
        FitSpec's x0 (n_iter_plain iterations) as the fallback; a voxel refitted plainly keeps the better
        (lower rms) of its two fits.

        judge="threshold": only voxels whose warm rms ends above `fallback_rms` (default 1.5 sigma, at
        least 1e-4) are refitted -- the fast rule. judge="plain": every voxel is also fitted plainly, so
        no voxel keeps a warm fit whose rms is above its plain fit's (costs the whole plain fit)."""
        import time
        from .fitting import fit
        if judge not in ("threshold", "plain"):
            raise ValueError(f"judge {judge!r}; use 'threshold' or 'plain'")
        z = np.atleast_2d(np.asarray(z_meas, np.float64))
        thr = fallback_rms if fallback_rms is not None else max(1.5 * self.sigma, 1e-4)
        t0 = time.perf_counter()
        x0 = self.starting_values(z)
        t1 = time.perf_counter()
        warm = fit(self.experiment, self.spec, z, n_iter=n_iter_warm, x0_phys=x0)
        t2 = time.perf_counter()
        x, rms = warm.x.copy(), warm.rms.copy()
        bad = np.flatnonzero(~(rms <= thr)) if judge == "threshold" else np.arange(z.shape[0])
        if bad.size:
            plain = fit(self.experiment, self.spec, z[bad], n_iter=n_iter_plain)
            better = ~(warm.rms[bad] <= plain.rms)
            x[bad[better]] = plain.x[better]
            rms[bad[better]] = plain.rms[better]
        t3 = time.perf_counter()
        refit = np.zeros(z.shape[0], bool)
        refit[bad] = True
        return WarmFitResult(x, rms, x0, refit, n_iter_warm, n_iter_plain,
                             {"predict": t1 - t0, "warm_lm": t2 - t1, "fallback": t3 - t2, "total": t3 - t0})
