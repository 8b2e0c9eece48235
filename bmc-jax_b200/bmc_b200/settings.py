"""Global precision switch, mirroring BMC-JAX `bmc_jax.settings` (settings.py:41-75).

`use_x64(True)` (the default here) runs forward simulations in float64; `use_x64(False)` selects the
float32 kernel. `use_precision("mixed")` selects the mixed kernel: float64 state and first Taylor term of every
sub-step, float32 for the later terms (BMC_MIXED in include/bmc_b200.h). Tangents, Jacobians and
fits always run in float64. `use_expm` is accepted for compatibility: both of the reference's backends
("library", "plain") compute the same matrix exponential, and this library has one kernel for it. No
environment variable is read.
"""
_STATE = {"precision": "f64", "expm": "library"}
EXPM_BACKENDS = ("library", "plain")
PRECISIONS = ("f64", "mixed", "f32")


def use_x64(enable: bool = True) -> bool:
    """Select float64 (True) or float32 (False) forward simulations. Returns the new state."""
    _STATE["precision"] = "f64" if enable else "f32"
    return x64_enabled()


def x64_enabled() -> bool:
    """True unless the float32 kernel is selected."""
    return _STATE["precision"] != "f32"


def use_precision(name: str = "f64") -> str:
    """Select the forward simulations' arithmetic: "f64", "mixed" or "f32"."""
    if name not in PRECISIONS:
        raise ValueError(f"use_precision: one of {PRECISIONS}, not {name!r}")
    _STATE["precision"] = name
    return name


def precision() -> str:
    return _STATE["precision"]


def use_expm(backend: str = "library") -> str:
    if backend not in EXPM_BACKENDS:
        raise ValueError(f"use_expm: one of {EXPM_BACKENDS}, not {backend!r}")
    _STATE["expm"] = backend
    return backend


def expm_backend() -> str:
    return _STATE["expm"]
