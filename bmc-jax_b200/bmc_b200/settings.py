"""Global precision switch, mirroring BMC-JAX `bmc_jax.settings` (settings.py:41-75).

`use_x64(True)` (the default here) runs forward simulations in float64; `use_x64(False)` selects the
float32 kernel. Tangents, Jacobians and fits always run in float64. `use_expm` is accepted for
compatibility: both of the reference's backends ("library", "plain") compute the same matrix
exponential, and this library has one kernel for it. No environment variable is read.
"""
_STATE = {"x64": True, "expm": "library"}
EXPM_BACKENDS = ("library", "plain")


def use_x64(enable: bool = True) -> bool:
    """Select float64 (True) or float32 (False) forward simulations. Returns the new state."""
    _STATE["x64"] = bool(enable)
    return x64_enabled()


def x64_enabled() -> bool:
    return bool(_STATE["x64"])


def use_expm(backend: str = "library") -> str:
    if backend not in EXPM_BACKENDS:
        raise ValueError(f"use_expm: one of {EXPM_BACKENDS}, not {backend!r}")
    _STATE["expm"] = backend
    return backend


def expm_backend() -> str:
    return _STATE["expm"]
