"""Saturation sequences built in code (BMC-JAX sequences/saturation.py:17-84); the Pulseq converter
(`events_from_seq`, `events_from_seq_batch`, `prep_rf_simulation`, module `pulseq`) is imported on
first use, as in BMC-JAX sequences/__init__.py:11-15."""
import numpy as np

from .simulation import EventType, SimEvent

__all__ = ["GAMMA_RAD_PER_S_UT", "GAMMA_HZ_PER_T", "hz_per_ppm", "cw_saturation", "events_from_seq",
           "events_from_seq_batch"]


def __getattr__(name):
    if name in ("events_from_seq", "events_from_seq_batch", "prep_rf_simulation", "read_seq"):
        from . import pulseq
        return getattr(pulseq, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")

#: Proton gyromagnetic ratio [rad / (s uT)]; /2pi gives 42.577 Hz/uT.
GAMMA_RAD_PER_S_UT = 267.5153
#: [Hz / T]
GAMMA_HZ_PER_T = 42.5764e6


def hz_per_ppm(b0_T: float) -> float:
    """Chemical-shift scale at this field [Hz/ppm]."""
    return GAMMA_HZ_PER_T * b0_T / 1e6


def cw_saturation(ppm, b1_uT: float, tsat_s: float, b0_T: float = 2.8936, m0_ppm=None) -> SimEvent:
    """One continuous-wave block of tsat_s at b1_uT per offset, then a zero-length ADC.

    Shape (n_offsets, 2); floating fields are float32 as the reference builds them. `m0_ppm`
    prepends one unsaturated reference offset."""
    ppm = np.atleast_1d(np.asarray(ppm, np.float64))
    if m0_ppm is not None:
        ppm = np.concatenate([[float(m0_ppm)], ppm])
    n = ppm.size
    if tsat_s < 0:
        raise ValueError(f"tsat_s must be >= 0, got {tsat_s}")
    if b1_uT < 0:
        raise ValueError(f"b1_uT must be >= 0, got {b1_uT}")
    amp_hz = b1_uT * GAMMA_RAD_PER_S_UT / (2 * np.pi)
    freq_hz = ppm * hz_per_ppm(b0_T)

    def pair(sat, adc):
        col = lambda v: np.full(n, v, np.float64) if np.isscalar(v) else np.asarray(v, np.float64)
        return np.stack([col(sat), col(adc)], axis=1)

    return SimEvent(type=pair(EventType.RF_PULSE, EventType.ADC).astype(np.int32),
                    dt=pair(tsat_s, 0.0).astype(np.float32),
                    rf_amp=pair(amp_hz, 0.0).astype(np.float32),
                    rf_phase=pair(0.0, 0.0).astype(np.float32),
                    rf_freq=pair(freq_hz, np.zeros(n)).astype(np.float32),
                    adc_idx=pair(-1, 0).astype(np.int32))
