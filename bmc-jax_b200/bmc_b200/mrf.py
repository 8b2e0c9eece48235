"""MR-fingerprinting dictionaries (BMC-JAX mrf/dictionary.py:22-111) on the voxel-batched kernel."""
from typing import Dict, Sequence, Tuple

import numpy as np

from .simulation import SimParams, SimEvent, simulate_z

__all__ = ["build_param_grid", "generate_dictionary"]


def build_param_grid(base_params: SimParams, grid: Dict[str, Sequence[float]]) -> SimParams:
    """The Cartesian product of `grid` as one batched SimParams (dictionary.py:22-66)."""
    if not grid:
        raise ValueError("grid must have at least one swept parameter")
    names = list(grid.keys())
    mesh = np.meshgrid(*[np.asarray(grid[n], np.float64) for n in names], indexing="ij")
    flat = [m.reshape(-1) for m in mesh]
    n = flat[0].shape[0]
    batched = SimParams(*[np.broadcast_to(np.asarray(v), (n,) + np.shape(v)) for v in base_params])
    upd = {}
    for name, values in zip(names, flat):
        shape = np.shape(getattr(base_params, name))
        if shape != () and any(s != 1 for s in shape):
            raise ValueError(f"Cannot sweep '{name}': base field has shape {shape} (more than one element). "
                             "Sweeping into a specific slot of a multi-pool field is not supported by "
                             "build_param_grid.")
        upd[name] = values.reshape((n,) + shape)
    return batched._replace(**upd)


def generate_dictionary(base_params: SimParams, seq_base: SimEvent, M_init, grid: Dict[str, Sequence[float]],
                        water_z_index: int, chunk_size: int = 20_000) -> Tuple[Dict[str, np.ndarray], np.ndarray]:
    """Fingerprints (n_entries, n_offsets) for every grid entry, `chunk_size` entries per launch
    (dictionary.py:69-111). Unlike the reference, only water Mz leaves the device."""
    pb = build_param_grid(base_params, grid)
    n = pb.water_r1.shape[0]
    entries = {name: np.asarray(getattr(pb, name)).reshape(-1) for name in grid}
    fp = np.empty((n, np.shape(seq_base.rf_amp)[0]), dtype=np.float32)
    for a in range(0, n, chunk_size):
        b = min(a + chunk_size, n)
        chunk = SimParams(*[np.asarray(v)[a:b] for v in pb])
        fp[a:b] = simulate_z(chunk, seq_base, np.broadcast_to(np.asarray(M_init), (b - a, np.size(M_init))),
                             water_z_index)
    return entries, fp
