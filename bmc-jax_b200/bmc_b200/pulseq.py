"""Pulseq `.seq` files -> event tables, without pypulseq (BMC-JAX sequences/pulseq.py:20-428).

`seq` is a `Sequence` from `read_seq`, a path to a `.seq` / `.seq.gz` file, or a pypulseq
`Sequence` (the converter reads only `block_events` and `get_block`). `read_seq` parses a Pulseq file
(format 1.4; 1.3 block delays are read too) into a `Sequence` whose `get_block(i)` exposes what the
reference's converter reads from a pypulseq block: `rf.signal` (complex, Hz), `rf.t`,
`rf.freq_offset`, `rf.phase_offset`, `rf.delay`, `gz`, `adc` and `block_duration`.
`events_from_seq`, `events_from_seq_batch` and `prep_rf_simulation` then follow the reference's
conversion rules step for step -- down-sampling of shaped pulses to `max_pulse_samples`, block pulses
longer than 0.1 s split into equal sub-steps, the frame phase accumulated per pulse from its frequency
offset and reset at every readout, spoilers from z gradients, one row per readout -- with the same
order of floating-point operations, so the tables it produces match the reference's shipped
conversions bit for bit (tests/test_pulseq.py).
"""
from __future__ import annotations

import gzip
from pathlib import Path
from types import SimpleNamespace
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import settings
from .simulation import EventType, SimEvent

__all__ = ["Sequence", "read_seq", "decompress_shape", "events_from_seq", "events_from_seq_batch",
           "prep_rf_simulation"]


def decompress_shape(packed: np.ndarray, num_samples: int) -> np.ndarray:
    """A Pulseq shape: run-length-encoded first differences (two equal values are followed by the
    count of further repeats), integrated by a cumulative sum. A shape whose stored length equals
    its sample count is stored uncompressed."""
    packed = np.asarray(packed, np.float64)
    if packed.size == num_samples:
        return packed.copy()
    out = np.empty(num_samples, np.float64)
    i = o = 0
    n = packed.size
    while i < n:
        if i + 1 < n and packed[i] == packed[i + 1]:
            rep = int(round(packed[i + 2])) + 2 if i + 2 < n else 2
            if o + rep > num_samples:
                raise ValueError(f"shape decompresses to more than {num_samples} samples")
            out[o:o + rep] = packed[i]
            o += rep
            i += 3
        else:
            if o >= num_samples:
                raise ValueError(f"shape decompresses to more than {num_samples} samples")
            out[o] = packed[i]
            o += 1
            i += 1
    if o != num_samples:
        raise ValueError(f"shape decompresses to {o} samples, header says {num_samples}")
    return np.cumsum(out)


class Sequence:
    """The parts of a Pulseq file the simulator needs (see the module notes)."""

    def __init__(self):
        self.version: Tuple[int, int, int] = (1, 4, 0)
        self.definitions: Dict[str, List[str]] = {}
        self.blocks: Dict[int, List[int]] = {}
        self.rf: Dict[int, List[float]] = {}
        self.grad: Dict[int, List[float]] = {}
        self.trap: Dict[int, List[float]] = {}
        self.adc: Dict[int, List[float]] = {}
        self.delays: Dict[int, float] = {}
        self.shapes: Dict[int, np.ndarray] = {}
        self._waves: Dict[tuple, SimpleNamespace] = {}

    @property
    def block_events(self) -> Dict[int, List[int]]:
        return self.blocks

    def raster(self, name: str, default: float) -> float:
        v = self.definitions.get(name)
        return float(v[0]) if v else default

    def shape(self, sid: int) -> np.ndarray:
        if sid not in self.shapes:
            raise ValueError(f"shape {sid} is referenced but not defined")
        return self.shapes[sid]

    def _waveform(self, amp, mag_id, ph_id, t_id) -> SimpleNamespace:
        """signal and sample times of an RF event; cached, as many events share one waveform."""
        key = (amp, mag_id, ph_id, t_id)
        w = self._waves.get(key)
        if w is None:
            mag = self.shape(mag_id)
            ph = self.shape(ph_id)
            if mag.size != ph.size:
                raise ValueError(f"RF shapes {mag_id} and {ph_id} differ in length")
            rf_raster = self.raster("RadiofrequencyRasterTime", 1e-6)
            w = SimpleNamespace(key=key, signal=amp * mag * np.exp(1j * 2 * np.pi * ph))
            if t_id == 0:
                w.t = (np.arange(1, mag.size + 1) - 0.5) * rf_raster
            else:
                w.t = self.shape(t_id) * rf_raster
            self._waves[key] = w
        return w

    def get_block(self, index: int) -> SimpleNamespace:
        """Block `index` (1-based): rf, gx, gy, gz, adc (None when absent) and block_duration [s]."""
        row = self.blocks[index]
        b = SimpleNamespace(rf=None, gx=None, gy=None, gz=None, adc=None)
        if self.version >= (1, 4, 0):
            b.block_duration = row[0] * self.raster("BlockDurationRaster", 1e-5)
            rf_id, gx, gy, gz, adc_id = row[1:6]
        else:                                   # format 1.3: the longest of the block's events
            delay_id, rf_id, gx, gy, gz, adc_id = row[0:6]
            durs = [self.delays.get(delay_id, 0.0)]
            for gid in (gx, gy, gz):
                if gid in self.trap:            # amp rise flat fall delay [us]
                    _, rise, flat, fall, gdelay = self.trap[gid][:5]
                    durs.append((gdelay + rise + flat + fall) * 1e-6)
            if adc_id:
                num, dwell, adelay = self.adc[adc_id][:3]
                durs.append(adelay * 1e-6 + num * dwell * 1e-9)
            b.block_duration = max(durs)
        if rf_id:
            amp, mag_id, ph_id, t_id, delay, freq, phase = self.rf[rf_id][:7]
            w = self._waveform(amp, int(mag_id), int(ph_id), int(t_id))
            b.rf = SimpleNamespace(signal=w.signal, t=w.t, waveform_key=w.key, delay=delay * 1e-6,
                                   freq_offset=freq, phase_offset=phase)
        for name, gid in (("gx", gx), ("gy", gy), ("gz", gz)):
            if gid:
                setattr(b, name, SimpleNamespace(id=gid))
        if adc_id:
            num, dwell, delay, freq, phase = self.adc[adc_id][:5]
            b.adc = SimpleNamespace(num_samples=int(num), dwell=dwell * 1e-9, delay=delay * 1e-6,
                                    freq_offset=freq, phase_offset=phase)
        return b


def _open(path):
    path = Path(path)
    if path.suffix == ".gz":
        return gzip.open(path, "rt")
    return open(path, "r")


def read_seq(path) -> Sequence:
    """Parse a Pulseq `.seq` file (plain or gzip-compressed)."""
    seq = Sequence()
    section = None
    shape_id = None
    shape_n = None
    shape_vals: List[float] = []

    def close_shape():
        if shape_id is not None:
            if shape_n is None:
                raise ValueError(f"shape {shape_id} has no num_samples line")
            seq.shapes[shape_id] = decompress_shape(np.asarray(shape_vals), shape_n)

    ver = {}
    with _open(path) as fh:
        for raw in fh:
            line = raw.strip()
            if not line or line.startswith("#"):
                continue
            if line.startswith("["):
                if section == "SHAPES":
                    close_shape()
                    shape_id = None
                section = line.strip("[]")
                continue
            tok = line.split()
            if section == "VERSION":
                ver[tok[0]] = int(tok[1])
            elif section == "DEFINITIONS":
                seq.definitions[tok[0]] = tok[1:]
            elif section == "BLOCKS":
                seq.blocks[int(tok[0])] = [int(x) for x in tok[1:]]
            elif section == "RF":
                seq.rf[int(tok[0])] = [float(x) for x in tok[1:]]
            elif section == "GRADIENTS":
                seq.grad[int(tok[0])] = [float(x) for x in tok[1:]]
            elif section == "TRAP":
                seq.trap[int(tok[0])] = [float(x) for x in tok[1:]]
            elif section == "ADC":
                seq.adc[int(tok[0])] = [float(x) for x in tok[1:]]
            elif section == "DELAYS":
                seq.delays[int(tok[0])] = float(tok[1]) * 1e-6
            elif section == "SHAPES":
                if tok[0] == "shape_id":
                    close_shape()
                    shape_id, shape_n, shape_vals = int(tok[1]), None, []
                elif tok[0] == "num_samples":
                    shape_n = int(tok[1])
                else:
                    shape_vals.append(float(tok[0]))
    if section == "SHAPES":
        close_shape()
    if ver:
        seq.version = (ver.get("major", 1), ver.get("minor", 4), ver.get("revision", 0))
    if sorted(seq.blocks) != list(range(1, len(seq.blocks) + 1)):
        raise ValueError("block numbers must run 1, 2, ... without gaps")
    return seq


# ------------------------------------------------------------------------------------------------
# conversion (sequences/pulseq.py:20-428)
# ------------------------------------------------------------------------------------------------
MAX_BLOCK_DT = 0.1            # block pulses longer than this are split into equal sub-steps [s]


def prep_rf_simulation(block, max_pulse_samples: int):
    """(amp, phase, dt, delay_after) of a block's RF: zero samples dropped (they become the delay after
    the pulse), block pulses collapsed to one sample, shaped pulses down-sampled to at most
    max_pulse_samples by keeping every f-th sample (sequences/pulseq.py:367-428)."""
    amp = np.abs(block.rf.signal)
    ph = np.angle(block.rf.signal)
    idx = np.argwhere(amp > 1e-6)
    rf_length = amp.size
    dtp = block.rf.t[1] - block.rf.t[0]
    delay_after = (rf_length - idx.size) * dtp
    amp = amp[idx]
    ph = ph[idx]
    n_unique = max(np.unique(amp).size, np.unique(ph).size)
    if n_unique == 1 and amp.size == 2:            # block pulse, format >= 1.4
        return amp[0], ph[0], dtp, delay_after
    if n_unique == 1:                              # block pulse, format < 1.4
        return amp[0], ph[0], dtp * amp.size, delay_after
    if amp.size > max_pulse_samples:
        f = int(np.ceil(amp.size / max_pulse_samples))
        return np.squeeze(amp[::f]), np.squeeze(ph[::f]), dtp * f, delay_after
    return np.squeeze(amp), np.squeeze(ph), dtp, delay_after


class _Rows:
    """Event columns being collected for one table row."""

    def __init__(self):
        self.type, self.dt, self.amp, self.phase, self.freq, self.adc = [], [], [], [], [], []

    def add(self, t, dt, amp=0.0, phase=0.0, freq=0.0, adc=-1):
        self.type.append(t)
        self.dt.append(dt)
        self.amp.append(amp)
        self.phase.append(phase)
        self.freq.append(freq)
        self.adc.append(adc)

    def extend(self, t, dt, amp, phase, freq):
        n = len(amp)
        self.type += [t] * n
        self.dt += [dt] * n
        self.amp += amp.tolist()
        self.phase += phase.tolist()
        self.freq += [freq] * n
        self.adc += [-1] * n

    def __len__(self):
        return len(self.type)


def _convert(seq, max_pulse_samples, split_at_adc):
    """Walk the blocks; a list of rows (one per readout when split_at_adc, else one)."""
    if max_pulse_samples <= 0:
        raise ValueError(f"max_pulse_samples must be positive, got {max_pulse_samples}")
    rows, cur = [], _Rows()
    current_adc = 0
    accum = 0.0
    prepared = {}                      # prep_rf_simulation depends on the waveform alone
    for bi in range(1, len(seq.block_events) + 1):
        block = seq.get_block(bi)
        if block.adc is not None:
            cur.add(EventType.ADC, 0.0, adc=current_adc)
            current_adc += 1
            accum = 0.0
            if split_at_adc:
                rows.append(cur)
                cur = _Rows()
                current_adc = 0
        elif block.rf is not None:
            key = getattr(block.rf, "waveform_key", None)
            prep = prepared.get(key) if key is not None else None
            if prep is None:
                prep = prep_rf_simulation(block, max_pulse_samples)
                if key is not None:
                    prepared[key] = prep
            amp, ph, dt, delay_after = prep
            phase_offset = float(block.rf.phase_offset)
            freq_offset = float(block.rf.freq_offset)
            start = accum
            phase_degree = float(dt) * amp.size * 360 * freq_offset
            accum += (phase_degree % 360) / 180 * np.pi
            if np.isscalar(amp) or amp.size == 1:
                total = float(dt)
                phase = -float(np.squeeze(ph)) + phase_offset - start
                freq = float(np.squeeze(block.rf.freq_offset))
                if total > MAX_BLOCK_DT:
                    n_sub = int(np.ceil(total / MAX_BLOCK_DT))
                    for _ in range(n_sub):
                        cur.add(EventType.RF_PULSE, total / n_sub, float(np.squeeze(amp)), phase, freq)
                else:
                    cur.add(EventType.RF_PULSE, total, float(np.squeeze(amp)), phase, freq)
            else:
                # the reference's per-sample loop, elementwise: (-ph + phase_offset) - start, in that order
                a = np.asarray(amp, np.float64).ravel()
                p = (-np.asarray(ph, np.float64).ravel() + phase_offset) - start
                cur.extend(EventType.RF_PULSE, float(dt), a, p, float(np.squeeze(block.rf.freq_offset)))
            if delay_after > 1e-12:
                cur.add(EventType.DELAY, float(delay_after))
        elif block.gz is not None:
            cur.add(EventType.SPOILER, float(block.block_duration))
        else:
            cur.add(EventType.DELAY, float(block.block_duration))
    if not split_at_adc:
        rows.append(cur)
    return rows


def _as_sequence(seq):
    return read_seq(seq) if isinstance(seq, (str, Path)) else seq


def events_from_seq(seq, max_pulse_samples: int = 500, max_events: Optional[int] = None):
    """The whole sequence as one event row (n_events,), padded to max_events with zero-length DELAYs
    (sequences/pulseq.py:20-183). Returns (SimEvent, n_events before padding); floats are float32,
    as the reference's."""
    row = _convert(_as_sequence(seq), max_pulse_samples, split_at_adc=False)[0]
    n = len(row)
    if max_events is not None:
        if n > max_events:
            raise ValueError(f"Sequence has {n} events, but max_events is {max_events}")
        for _ in range(max_events - n):
            row.add(EventType.DELAY, 0.0)
    ev = SimEvent(np.asarray(row.type, np.int32), np.asarray(row.dt, np.float32), np.asarray(row.amp, np.float32),
                  np.asarray(row.phase, np.float32), np.asarray(row.freq, np.float32), np.asarray(row.adc, np.int32))
    return ev, n


def events_from_seq_batch(seq, max_pulse_samples: int = 500):
    """One row per readout (every ADC ends a row), zero-padded at the back to the longest
    (sequences/pulseq.py:185-365). Returns (SimEvent (n_rows, n_events), n_rows); floats are float64
    when x64 is enabled, else float32, as `jnp.array` of the reference's float64 arrays."""
    rows = _convert(_as_sequence(seq), max_pulse_samples, split_at_adc=True)
    n = len(rows)
    width = max((len(r) for r in rows), default=0)
    t = np.zeros((n, width), np.int32)
    dt = np.zeros((n, width))
    amp = np.zeros((n, width))
    ph = np.zeros((n, width))
    fr = np.zeros((n, width))
    adc = np.full((n, width), -1, np.int32)
    for i, r in enumerate(rows):
        k = len(r)
        t[i, :k], dt[i, :k], amp[i, :k], ph[i, :k], fr[i, :k], adc[i, :k] = r.type, r.dt, r.amp, r.phase, r.freq, r.adc
    real = np.float64 if settings.x64_enabled() else np.float32
    return SimEvent(t, dt.astype(real), amp.astype(real), ph.astype(real), fr.astype(real), adc), n
