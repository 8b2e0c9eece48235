"""Pulseq reader and converter (bmc_b200.pulseq) against the reference's own conversions.

The reference ships its 14 phantom sequences both as Pulseq files (examples/data/seqs/*.seq, here
gzip-compressed) and as the event tables its converter made from them (examples/data/events/*.npz,
max_pulse_samples = 200). Converting the files here must reproduce those tables bit for bit. A small
hand-written file then covers the rules those sequences do not reach (block pulses split into 0.1 s
sub-steps, zero samples becoming a trailing delay, down-sampling, phase accumulation and its reset
at readouts, padding), with values worked out by hand from the reference's rules
(sequences/pulseq.py:20-428).
"""
import gzip
from pathlib import Path

import numpy as np
import pytest

import bmc_oracle as O
from bmc_b200 import settings
from bmc_b200.pulseq import decompress_shape, events_from_seq, events_from_seq_batch, read_seq
from bmc_b200.simulation import EventType, SimEvent
from conftest import GOLDEN

PHANTOM = GOLDEN / "phantom"
STEMS = sorted(p.name[:-len(".seq.gz")] for p in (PHANTOM / "seqs").glob("*.seq.gz"))
FIELDS = SimEvent._fields


def test_fixture_set_is_complete():
    assert len(STEMS) == 14
    assert {s + "_events.npz" for s in STEMS} <= {p.name for p in PHANTOM.glob("*_events.npz")}


@pytest.mark.parametrize("stem", STEMS)
def test_shipped_sequences_convert_bit_for_bit(stem):
    d = np.load(PHANTOM / f"{stem}_events.npz")
    ev, n = events_from_seq_batch(PHANTOM / "seqs" / f"{stem}.seq.gz", max_pulse_samples=int(d["max_pulse_samples"]))
    assert n == int(d["n_batches"])
    for f in FIELDS:
        got, want = np.asarray(getattr(ev, f)), d[f]
        assert got.dtype == want.dtype, f
        np.testing.assert_array_equal(got, want, err_msg=f)


def test_decompress_shape():
    # first differences 0.125 x 8, -1, 0 x 7: "v v n" means v repeated n + 2 times
    mag = decompress_shape(np.array([0.125, 0.125, 6, -1, 0, 0, 5]), 16)
    np.testing.assert_array_equal(mag, np.r_[np.arange(1, 9) * 0.125, np.zeros(8)])
    np.testing.assert_array_equal(decompress_shape(np.array([3.0, 4.0]), 2), [3.0, 4.0])   # stored raw
    with pytest.raises(ValueError, match="header says"):
        decompress_shape(np.array([0.5, 0.5, 1]), 4)
    with pytest.raises(ValueError, match="more than"):
        decompress_shape(np.array([0.5, 0.5, 9]), 4)


SEQ = """# hand-written Pulseq file
[VERSION]
major 1
minor 4
revision 2

[DEFINITIONS]
AdcRasterTime 1e-07
BlockDurationRaster 1e-05
GradientRasterTime 1e-05
RadiofrequencyRasterTime 1e-06

# NUM DUR RF GX GY GZ ADC EXT
[BLOCKS]
1 100000 0 0 0 0 0 0
2 25000 1 0 0 0 0 0
3 100 0 0 0 1 0 0
4 2 2 0 0 0 0 0
5 1 0 0 0 0 1 0
6 25000 3 0 0 0 0 0
7 1 0 0 0 0 1 0

# id amplitude mag_id phase_id time_shape_id delay freq phase
[RF]
1 42.5764 1 2 3 0 123.25 0.5
2 100 4 5 0 0 -50 0
3 21.2882 1 2 3 0 -400 0

# id amplitude rise flat fall delay
[TRAP]
1 1000 100 800 100 0

# id num dwell delay freq phase
[ADC]
1 1 10000 0 0 0

[SHAPES]

shape_id 1
num_samples 2
1
1

shape_id 2
num_samples 2
0
0

shape_id 3
num_samples 2
0
250000

shape_id 4
num_samples 16
0.125
0.125
6
-1
0
0
5

shape_id 5
num_samples 16
0.125
0
0
5
-0.125
0
0
5
"""


@pytest.fixture
def seq_path(tmp_path):
    p = tmp_path / "hand.seq"
    p.write_text(SEQ)
    gz = tmp_path / "hand.seq.gz"
    with gzip.open(gz, "wt") as fh:
        fh.write(SEQ)
    return p, gz


def _expected_rows():
    """The two readout rows of SEQ by the reference's rules, worked out by hand."""
    RF, DL, SP, AD = EventType.RF_PULSE, EventType.DELAY, EventType.SPOILER, EventType.ADC
    # block 2: 0.25 s block pulse (> 0.1 s) -> 3 equal sub-steps; phase = -0 + 0.5 - 0 (nothing accumulated yet)
    # it advances the frame by (0.25 * 1 * 360 * 123.25) mod 360 = 292.5 degrees
    start = 292.5 / 180 * np.pi
    # block 4: 16 samples at the raster midpoints, the last 8 zero -> 8 steps + a delay of 8 samples
    t = (np.arange(1, 17) - 0.5) * 1e-6
    dtp = t[1] - t[0]
    ang = float(np.angle(np.exp(1j * 2 * np.pi * 0.125)))           # phase shape 0.125 cycles
    row1 = [(DL, 100000 * 1e-5, 0, 0, 0, -1)]
    row1 += [(RF, 0.25 / 3, 42.5764, 0.5, 123.25, -1)] * 3
    row1 += [(SP, 100 * 1e-5, 0, 0, 0, -1)]
    row1 += [(RF, dtp, 100 * 0.125 * k, -ang + 0.0 - start, -50.0, -1) for k in range(1, 9)]
    row1 += [(DL, 8 * dtp, 0, 0, 0, -1), (AD, 0, 0, 0, 0, 0)]
    # the readout resets the frame: block 6 starts from phase 0 again
    row2 = [(RF, 0.25 / 3, 21.2882, 0.0, -400.0, -1)] * 3 + [(AD, 0, 0, 0, 0, 0)]
    return row1, row2


def _cols(rows, width):
    out = [np.zeros(width, np.int32)] + [np.zeros(width) for _ in range(4)] + [np.full(width, -1, np.int32)]
    for j, r in enumerate(rows):
        for c in range(6):
            out[c][j] = r[c]
    return out


def test_hand_written_sequence_batch(seq_path):
    row1, row2 = _expected_rows()
    for path in seq_path:
        ev, n = events_from_seq_batch(path, max_pulse_samples=200)
        assert n == 2 and ev.dt.shape == (2, len(row1))
        for i, rows in enumerate((row1, row2)):
            want = _cols(rows, len(row1))             # row 2 zero-padded at the back (DELAY, dt 0, adc -1)
            for c, f in enumerate(FIELDS):
                np.testing.assert_allclose(getattr(ev, f)[i], want[c], rtol=0, atol=1e-15, err_msg=f"row {i} {f}")
    # all but the phases of the shaped pulse are exact
    np.testing.assert_array_equal(ev.dt[0], _cols(row1, len(row1))[1])
    np.testing.assert_array_equal(ev.rf_amp[0], _cols(row1, len(row1))[2])


def test_hand_written_sequence_single_row_and_padding(seq_path):
    row1, row2 = _expected_rows()
    rows = row1 + [r[:5] + ((1,) if r[0] == EventType.ADC else (-1,)) for r in row2]   # readouts numbered on
    ev, n = events_from_seq(seq_path[0], max_pulse_samples=200)
    assert n == len(rows) and ev.dt.dtype == np.float32 and ev.type.dtype == np.int32
    want = _cols(rows, len(rows))
    for c, f in enumerate(FIELDS):
        np.testing.assert_allclose(getattr(ev, f), np.asarray(want[c]).astype(getattr(ev, f).dtype), rtol=0,
                                   atol=0, err_msg=f)
    ev, n2 = events_from_seq(seq_path[0], max_pulse_samples=200, max_events=n + 5)
    assert n2 == n and ev.dt.shape == (n + 5,)
    assert (ev.type[n:] == EventType.DELAY).all() and (ev.dt[n:] == 0).all() and (ev.adc_idx[n:] == -1).all()
    with pytest.raises(ValueError, match="max_events is"):
        events_from_seq(seq_path[0], max_pulse_samples=200, max_events=n - 1)


def test_down_sampling_keeps_every_fth_sample(seq_path):
    ev, _ = events_from_seq_batch(seq_path[0], max_pulse_samples=3)
    t = (np.arange(1, 17) - 0.5) * 1e-6
    dtp = t[1] - t[0]
    shaped = (ev.type[0] == EventType.RF_PULSE) & (ev.rf_freq[0] == -50.0)
    # 8 samples > 3 -> every ceil(8 / 3) = 3rd sample, each 3 raster steps long
    np.testing.assert_array_equal(ev.rf_amp[0][shaped], [12.5, 50.0, 87.5])
    np.testing.assert_array_equal(ev.dt[0][shaped], [dtp * 3] * 3)
    with pytest.raises(ValueError, match="max_pulse_samples"):
        events_from_seq_batch(seq_path[0], max_pulse_samples=0)


def test_float32_without_x64(seq_path):
    settings.use_x64(False)
    try:
        ev, _ = events_from_seq_batch(seq_path[0], max_pulse_samples=200)
        assert ev.dt.dtype == np.float32 and ev.type.dtype == np.int32
    finally:
        settings.use_x64(True)


def test_lazy_export_and_malformed_files(tmp_path):
    from bmc_b200 import sequences
    assert sequences.events_from_seq_batch is events_from_seq_batch
    bad = tmp_path / "gap.seq"
    bad.write_text("[BLOCKS]\n1 10 0 0 0 0 0 0\n3 10 0 0 0 0 0 0\n")
    with pytest.raises(ValueError, match="without gaps"):
        read_seq(bad)
    bad.write_text(SEQ.replace("shape_id 5", "shape_id 6"))
    with pytest.raises(ValueError, match="shape 5"):
        events_from_seq_batch(bad)


def test_block_pulse_file_simulates_like_cw_saturation(tmp_path):
    """A CW saturation written as Pulseq block pulses (how the reference's example 03 builds it) converts
    to 20 sub-steps of 0.1 s per offset; the oracle gives the same Z as for the single CW block."""
    from bmc_b200.sequences import cw_saturation
    ppm, b1, tsat, b0 = np.array([-3.0, 0.0, 2.0]), 1.0, 2.0, 3.0
    cw = cw_saturation(ppm, b1, tsat, b0)
    amp, freq = cw.rf_amp[:, 0].astype(np.float64), cw.rf_freq[:, 0].astype(np.float64)
    blocks = "".join(f"{2 * i + 1} {int(round(tsat / 1e-5))} {i + 1} 0 0 0 0 0\n{2 * i + 2} 1 0 0 0 0 1 0\n"
                     for i in range(ppm.size))
    rfs = "".join(f"{i + 1} {float(amp[i])!r} 1 2 3 0 {float(freq[i])!r} 0\n" for i in range(ppm.size))
    text = (f"[VERSION]\nmajor 1\nminor 4\nrevision 2\n[DEFINITIONS]\nBlockDurationRaster 1e-05\n"
            f"RadiofrequencyRasterTime 1e-06\n[BLOCKS]\n{blocks}[RF]\n{rfs}[ADC]\n1 1 10000 0 0 0\n[SHAPES]\n"
            f"shape_id 1\nnum_samples 2\n1\n1\nshape_id 2\nnum_samples 2\n0\n0\n"
            f"shape_id 3\nnum_samples 2\n0\n{int(round(tsat / 1e-6))}\n")
    path = tmp_path / "cw.seq"
    path.write_text(text)
    ev, n = events_from_seq_batch(path, max_pulse_samples=200)
    assert n == 3 and ev.dt.shape == (3, 21)
    np.testing.assert_array_equal(ev.dt[:, :20], tsat / 20)
    np.testing.assert_array_equal(ev.rf_amp[:, :20], np.repeat(amp[:, None], 20, 1))
    np.testing.assert_array_equal(ev.rf_phase, 0.0)
    p = O.make_params(1 / 1.3, 1 / 0.08, [500.0], [0.002], [3.5], [1.0], [30.0], b0=b0)
    m0 = O.initial_state(p)
    mz = O.mz_loc(1)
    z_seq = O.simulate_spectrum(p, O.Events(*ev), m0)[:, mz]
    z_cw = O.simulate_spectrum(p, O.Events(*[np.asarray(a, np.float64) if a.dtype.kind == "f" else a for a in cw]),
                               m0)[:, mz]
    np.testing.assert_allclose(z_seq, z_cw, rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_converted_table_on_the_gpu_matches_the_oracle(cuda):
    """A converted phantom sequence through the CUDA path, against the C oracle on the same table."""
    from bmc_b200.configs import example_config
    from bmc_b200.simulation import initial_state, pack_params, simulate_z, to_sim_params
    params = example_config("amide")
    p = to_sim_params(params)
    ev, n = events_from_seq_batch(PHANTOM / "seqs" / "quest_sim_tsat_1s.seq.gz", max_pulse_samples=200)
    m0 = np.asarray(initial_state(p))
    z = simulate_z(p, ev, m0, params.mz_loc)
    nc = int(np.shape(p.cest_k)[-1])
    want = O.c_simulate_z(pack_params(p, 1), O.Events(*ev), m0[None], nc, params.mz_loc)[0]
    np.testing.assert_allclose(np.asarray(z).reshape(-1), want, rtol=0, atol=1e-10)
