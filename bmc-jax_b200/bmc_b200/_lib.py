"""ctypes binding of libbmc_b200.so (the C ABI in include/bmc_b200.h).

The library is built in-tree (bmc-jax_b200/build.py) next to this file. There is no fallback: if
the shared library or a CUDA device is missing, every simulation or fit raises.
Device memory and streams come from torch (plumbing only); every call is asynchronous on the
current torch stream.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_NAME = "libbmc_b200.so"
LIB_PATH = Path(__file__).resolve().parent / LIB_NAME

MAX_CEST = 5
MAX_TANGENTS = 8
F64, F32, MIXED = 0, 1, 2
SEED_NONE, SEED_SPREAD_SIGMA = -1, -2
SLOT_SPREAD_SIGMA, SLOT_M_START = -2, -3
TANGENTS_AUTO, TANGENTS_FORWARD = 0, 1

EXPORTS = ("bmc_abi_version", "bmc_version", "bmc_last_error", "bmc_release", "bmc_simulate",
           "bmc_simulate_jvp", "bmc_simulate_design_jvp", "bmc_simulate_trajectory", "bmc_lm_fit", "bmc_normal_blocks",
           "bmc_simulate_counted", "bmc_simulate_jvp_counted", "bmc_probe_fma_peak", "bmc_simulate_noalloc",
           "bmc_mlp_sizes", "bmc_mlp_sync", "bmc_mlp_forward", "bmc_mlp_backward", "bmc_mlp_adam_step",
           "bmc_mlp_adam_step_dev", "bmc_uneven_uses_block_kernel", "bmc_uneven_create", "bmc_uneven_simulate",
           "bmc_uneven_destroy", "bmc_uneven_set_dense_switch", "bmc_normal_segments", "bmc_schur_step", "bmc_schur_eliminate", "bmc_schur_back",
           "bmc_set_tangent_mode")


class Problem(C.Structure):
    _fields_ = [("n_voxels", C.c_int32), ("n_offsets", C.c_int32), ("n_events", C.c_int32),
                ("n_cest", C.c_int32), ("mz_loc", C.c_int32), ("reset_after_adc", C.c_int32),
                ("precision", C.c_int32), ("reserved", C.c_int32)]


class Events(C.Structure):
    _fields_ = [("d_type", C.c_void_p), ("d_dt", C.c_void_p), ("d_rf_amp", C.c_void_p),
                ("d_rf_phase", C.c_void_p), ("d_rf_freq", C.c_void_p), ("d_adc_idx", C.c_void_p)]


class Spread(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("h_u", C.POINTER(C.c_double)), ("h_w", C.POINTER(C.c_double)),
                ("d_sigma_hz", C.c_void_p)]


class Tangents(C.Structure):
    _fields_ = [("n_tangents", C.c_int32), ("field_row", C.c_int32 * MAX_TANGENTS),
                ("d_seed", C.c_void_p), ("d_dm0", C.c_void_p)]


class FitSpecC(C.Structure):
    _fields_ = [("n_params", C.c_int32), ("n_iter", C.c_int32), ("lam0", C.c_double),
                ("field_row", C.c_int32 * MAX_TANGENTS), ("mode", C.c_int32 * MAX_TANGENTS),
                ("scale", C.c_double * MAX_TANGENTS), ("lo", C.c_double * MAX_TANGENTS),
                ("hi", C.c_double * MAX_TANGENTS), ("d_free", C.c_void_p),
                ("n_points_skip", C.c_int32), ("reserved", C.c_int32)]


class TableSet(C.Structure):
    _fields_ = [("n_tables", C.c_int32), ("h_n_offsets", C.POINTER(C.c_int32)), ("h_n_events", C.POINTER(C.c_int32)),
                ("ev", Events)]


class MlpShape(C.Structure):
    _fields_ = [("n_in", C.c_int32), ("n_hidden", C.c_int32), ("n_hidden_layers", C.c_int32), ("n_out", C.c_int32)]


_lib = None


def lib():
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python bmc-jax_b200/build.py` "
                               "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        L.bmc_abi_version.restype = C.c_int32
        L.bmc_version.restype = C.c_char_p
        L.bmc_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.bmc_last_error.restype = C.c_size_t
        L.bmc_release.restype = C.c_int
        L.bmc_simulate.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, C.POINTER(Spread), vp, vp]
        L.bmc_simulate.restype = C.c_int
        L.bmc_simulate_jvp.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, C.POINTER(Spread),
                                       C.POINTER(Tangents), vp, vp, vp]
        L.bmc_simulate_jvp.restype = C.c_int
        L.bmc_simulate_design_jvp.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, vp, C.POINTER(Events), vp,
                                              C.POINTER(Tangents), vp, vp, vp, vp, vp]
        L.bmc_simulate_design_jvp.restype = C.c_int
        L.bmc_simulate_trajectory.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, vp, vp]
        L.bmc_simulate_trajectory.restype = C.c_int
        L.bmc_lm_fit.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, C.POINTER(Spread),
                                 C.POINTER(FitSpecC), vp, vp, vp, vp, vp, vp]
        L.bmc_lm_fit.restype = C.c_int
        L.bmc_normal_blocks.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp]
        L.bmc_normal_blocks.restype = C.c_int
        L.bmc_simulate_counted.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, C.POINTER(Spread), vp,
                                           vp, vp]
        L.bmc_simulate_counted.restype = C.c_int
        L.bmc_simulate_jvp_counted.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, C.POINTER(Spread),
                                               C.POINTER(Tangents), vp, vp, vp, vp]
        L.bmc_simulate_jvp_counted.restype = C.c_int
        L.bmc_probe_fma_peak.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double), vp]
        L.bmc_probe_fma_peak.restype = C.c_int
        L.bmc_set_tangent_mode.argtypes = [C.c_int32]
        L.bmc_set_tangent_mode.restype = C.c_int
        L.bmc_simulate_noalloc.argtypes = [C.POINTER(Problem), vp, C.POINTER(Events), vp, C.POINTER(Spread), vp, vp]
        L.bmc_simulate_noalloc.restype = C.c_int
        i32p = C.POINTER(C.c_int32)
        L.bmc_uneven_create.argtypes = [C.c_int32, C.c_int32, i32p, C.POINTER(TableSet), C.c_int32, C.c_int32,
                                        C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.bmc_uneven_simulate.argtypes = [vp, vp, vp, C.POINTER(Spread), C.POINTER(Tangents), vp, vp, vp, vp]
        L.bmc_uneven_destroy.argtypes = [vp]
        L.bmc_uneven_set_dense_switch.argtypes = [vp, C.c_double]
        L.bmc_uneven_uses_block_kernel.argtypes = [vp, C.POINTER(C.c_int32)]
        L.bmc_normal_segments.argtypes = [C.c_int32, C.c_int32, C.c_int64, vp, vp, vp, vp, vp, vp, vp]
        L.bmc_schur_step.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, C.c_double, vp, vp, vp, vp, vp]
        L.bmc_schur_eliminate.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, C.c_double, vp, vp, vp, vp]
        L.bmc_schur_back.argtypes = [C.c_int32, C.c_int32, C.c_int32, vp, C.c_double, vp, vp, vp, vp, vp]
        for f in ("bmc_uneven_create", "bmc_uneven_simulate", "bmc_uneven_destroy", "bmc_uneven_set_dense_switch",
                  "bmc_uneven_uses_block_kernel", "bmc_normal_segments",
                  "bmc_schur_step", "bmc_schur_eliminate", "bmc_schur_back"):
            getattr(L, f).restype = C.c_int
        sp, i64p = C.POINTER(MlpShape), C.POINTER(C.c_int64)
        L.bmc_mlp_sizes.argtypes = [sp, C.c_int64, i64p, i64p, i64p]
        L.bmc_mlp_sync.argtypes = [sp, vp, vp, vp]
        L.bmc_mlp_forward.argtypes = [sp, vp, vp, vp, vp, vp, C.c_int64, vp, vp, C.c_int32, vp]
        L.bmc_mlp_backward.argtypes = [sp, vp, vp, C.c_int64, vp, vp, vp, vp]
        L.bmc_mlp_adam_step.argtypes = [sp, vp, vp, vp, vp, vp, C.c_int32, C.c_float, C.c_float, C.c_float,
                                        C.c_float, vp]
        L.bmc_mlp_adam_step_dev.argtypes = [sp, vp, vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float,
                                            vp]
        for f in ("bmc_mlp_sizes", "bmc_mlp_sync", "bmc_mlp_forward", "bmc_mlp_backward", "bmc_mlp_adam_step",
                  "bmc_mlp_adam_step_dev"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        buf = C.create_string_buffer(1024)
        lib().bmc_last_error(buf, 1024)
        raise RuntimeError(f"bmc_b200 error {status}: {buf.value.decode(errors='replace')}")


def torch_cuda():
    """torch, with a CUDA device required (the product path has no CPU fallback)."""
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("bmc_b200 needs a CUDA device (B200, sm_100a); none is available")
    return torch


def ptr(t) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def stream_handle():
    torch = torch_cuda()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def spread_struct(u, w, sigma_dev):
    """(struct, keep-alive) for a B0 spread, or (None, None)."""
    if u is None:
        return None, None
    u = np.ascontiguousarray(u, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    s = Spread(int(u.size), u.ctypes.data_as(C.POINTER(C.c_double)), w.ctypes.data_as(C.POINTER(C.c_double)),
               sigma_dev.data_ptr())
    return s, (u, w, sigma_dev)
