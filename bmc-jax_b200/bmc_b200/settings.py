"""Global precision switch, mirroring BMC-JAX `bmc_jax.settings` (settings.py:41-75).

`use_x64(True)` (the default here) runs forward simulations in float64; `use_x64(False)` selects the
float32 kernel. `use_precision("mixed")` selects the mixed kernel: float64 state and first Taylor term of every
sub-step, float32 for the later terms (BMC_MIXED in include/bmc_b200.h). Tangents, Jacobians and
fits always run in float64. `use_expm` is accepted for compatibility: both of the reference's backends
("library", "plain") compute the same matrix exponential, and this library has one kernel for it.
`use_tangents("forward")` keeps Jacobians in forward mode (one dual-number launch per tangent) where
"auto" (the default) computes every tangent of a single-event table -- CW Z-spectra, B1 ladders -- from
one Frechet derivative of the exponential (bmc_set_tangent_mode in include/bmc_b200.h); both give the same
derivatives to rounding. No environment variable is read.
"""
_STATE = {"precision": "f64", "expm": "library", "tangents": "auto"}
EXPM_BACKENDS = ("library", "plain")
PRECISIONS = ("f64", "mixed", "f32")
TANGENT_MODES = ("auto", "forward")


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


def use_tangents(mode: str = "auto") -> str:
    """Select how Jacobians are computed: "auto" or "forward" (process-wide, in the library)."""
    if mode not in TANGENT_MODES:
        raise ValueError(f"use_tangents: one of {TANGENT_MODES}, not {mode!r}")
    from . import _lib
    _lib.check(_lib.lib().bmc_set_tangent_mode(_lib.TANGENTS_AUTO if mode == "auto" else _lib.TANGENTS_FORWARD))
    _STATE["tangents"] = mode
    return mode


def tangent_mode() -> str:
    return _STATE["tangents"]
