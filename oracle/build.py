"""Build the C oracle (test infrastructure): oracle/_build/liboracle.so, gcc -O3 -fopenmp.

    python oracle/build.py
"""
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "liboracle.so"


def build(force=False):
    src = HERE / "bmc_oracle.c"
    if not force and OUT.exists() and OUT.stat().st_mtime > src.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-o", str(OUT), str(src), "-lm"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
