"""Build recipe of the oracle library (test infrastructure only).

``python oracle/build.py`` compiles ``krr_oracle.cpp`` into ``oracle/libkrr_oracle.so``
with g++, OpenMP and no floating-point contraction (the reference kernel is compiled
with ``fastmath=False``), so that each product and sum rounds separately.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "krr_oracle.cpp"
LIB = HERE / "libkrr_oracle.so"

FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
         "-fno-finite-math-only", "-Wall", "-Wextra", "-Wno-unused-parameter"]


def build(force: bool = False) -> Path:
    """Compile the oracle library if it is missing or older than its source; return its path."""
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(f".so.{os.getpid()}.tmp")  # per process: concurrent builds must not share it
    cmd = ["g++", *FLAGS, str(SRC), "-o", str(tmp)]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
