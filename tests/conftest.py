"""Shared test setup: the `gpu` marker, import paths, golden fixtures."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "bmc-jax_b200"))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libbmc_b200.so")


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


def unpack_params(d, prefix, cls):
    from bmc_oracle import FIELDS
    return cls(*[np.asarray(d[prefix + f]) for f in FIELDS])


def unpack_events(d, prefix, cls):
    return cls(*[np.asarray(d[prefix + f]) for f in ("type", "dt", "rf_amp", "rf_phase", "rf_freq", "adc_idx")])


@pytest.fixture(scope="session")
def cuda():
    """Skip-free GPU gate: `-m gpu` runs only where a GPU exists; on one, a missing library fails."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device (run with -m 'not gpu' on CPU)")
    import bmc_b200
    bmc_b200._load_library()
    return torch
