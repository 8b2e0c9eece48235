"""The benchmark's reference arm (`bench.py --impl reference`) on the host: it times the CPU oracle on
a bounded sample of the forward workload and prints one JSON line in the benchmark's format; under
torchrun only rank 0 prints, the other ranks exit 0 without work. Run on a small workload (11
offsets, one pulse) so that it takes seconds."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
ARGS = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-budget", "1", "--offsets", "11",
        "--pulses", "1", "--voxels", "4"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *ARGS], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_the_benchmark_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "Z-spectra/s (batched forward simulation)"
    assert line["unit"] == "Z-spectra/s" and line["higher_is_better"] is True
    assert line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and "voxels" in cb["sample"]
    assert cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
