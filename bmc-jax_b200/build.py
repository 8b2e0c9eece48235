"""Build libbmc_b200.so for sm_100a, in-tree (next to the Python package that loads it).

    python bmc-jax_b200/build.py [--force]

nvcc cross-compiles without a GPU. The library is rebuilt when any source under csrc/ or the
public header is newer than it.
"""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
OUT = HERE / "bmc_b200" / "libbmc_b200.so"
HEADER = HERE.parent / "include" / "bmc_b200.h"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC,-O2", "-shared", "--expt-relaxed-constexpr"]


def sources():
    return sorted(SRC.glob("*.cu"))


def stale() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = list(SRC.glob("*.cu")) + list(SRC.glob("*.cuh")) + [HEADER]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return OUT
    cmd = [NVCC, *FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-o", str(OUT), *map(str, sources())]
    print(" ".join(cmd), flush=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd[cmd.index("-o") + 1] = str(tmp)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", OUT)
