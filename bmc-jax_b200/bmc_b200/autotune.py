"""Measured tuning of uneven plans: the norm above which an event takes the dense path.

An event whose generator norm ||X|| = dt ||A|| is large is exponentiated densely -- a lane group per chain,
scaling and squaring -- and a smaller one by the truncated Taylor action, one lane per chain. Both meet
the same tolerance; which is faster depends on the pool count (the group's lanes, the sparse operator's
cost) and on the tables' events. `tune_dense_switch` times one forward pass of every pool-count group of
an UnevenBatch for each candidate threshold (CUDA events, after a warm-up pass), keeps the fastest, and
can store the choices in a JSON file that `apply_tuning` reads back for a batch of the same shapes.
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib

__all__ = ["tune_dense_switch", "apply_tuning", "plan_key", "uses_block_kernel"]

DEFAULT_CANDIDATES = (3.0, 6.0, 12.0, 25.0, 50.0, 100.0)


def plan_key(group) -> str:
    """A key for a pool-count group of an UnevenBatch: its pool count and a digest of its tables' sizes
    and of which table every voxel uses."""
    h = hashlib.sha1()
    h.update(np.asarray(group.plan.n_rows, np.int64).tobytes())
    h.update(np.asarray(group.plan.vox_table, np.int64).tobytes())
    return f"nc{group.nc}-{h.hexdigest()[:16]}"


def _set(group, norm: float) -> None:
    _lib.check(_lib.lib().bmc_uneven_set_dense_switch(group.plan.plan, float(norm)))


def uses_block_kernel(group) -> bool:
    """True when the group's plan takes the block kernel (every row one repeated block, automatic tangent
    mode): all its events are then exponentiated densely and the threshold is not consulted."""
    import ctypes as C
    out = C.c_int32(0)
    _lib.check(_lib.lib().bmc_uneven_uses_block_kernel(group.plan.plan, C.byref(out)))
    return bool(out.value)


def _time_pass(group, repeats: int) -> float:
    torch = _lib.torch_cuda()
    z = torch.empty(group.n_chains, dtype=torch.float64, device="cuda")
    group.plan.run(group.params, group.m0, z=z)                 # warm-up
    best = float("inf")
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        group.plan.run(group.params, group.m0, z=z)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune_dense_switch(batch, candidates: Sequence[float] = DEFAULT_CANDIDATES, repeats: int = 2,
                      path: Optional[str] = None) -> Dict[str, dict]:
    """For every pool-count group of `batch`, time one forward pass per candidate threshold, set the
    fastest on the group's plan and return {key: {"dense_switch": best, "ms": {candidate: ms}}}; with
    `path`, merge the choices into that JSON file. A group whose plan takes the block kernel
    (uses_block_kernel) has no threshold to tune: it gets {"dense_switch": None, "block_kernel": True}."""
    out: Dict[str, dict] = {}
    for g in batch.groups:
        if uses_block_kernel(g):
            out[plan_key(g)] = {"dense_switch": None, "block_kernel": True, "ms": {}, "voxels": int(len(g.voxels)),
                                "chains": int(g.n_chains)}
            continue
        ms = {}
        for c in candidates:
            _set(g, c)
            ms[float(c)] = _time_pass(g, repeats)
        best = min(ms, key=ms.get)
        _set(g, best)
        out[plan_key(g)] = {"dense_switch": best, "ms": ms, "voxels": int(len(g.voxels)),
                            "chains": int(g.n_chains)}
    if path is not None:
        p = Path(path)
        stored = json.loads(p.read_text()) if p.exists() else {}
        stored.update({k: {**v, "ms": {str(c): t for c, t in v["ms"].items()}} for k, v in out.items()})
        p.write_text(json.dumps(stored, indent=1, sort_keys=True))
    return out


def apply_tuning(batch, path: str) -> Dict[str, float]:
    """Set the stored threshold on every group of `batch` whose key is in the JSON file at `path`; returns
    {key: threshold} of the groups it set (the others keep the library's default)."""
    stored = json.loads(Path(path).read_text())
    done = {}
    for g in batch.groups:
        k = plan_key(g)
        if k in stored and stored[k].get("dense_switch") is not None:
            _set(g, stored[k]["dense_switch"])
            done[k] = float(stored[k]["dense_switch"])
    return done
