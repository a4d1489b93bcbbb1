"""Build the CUDA library ``kerrray_b200/libkerrray_cuda.so`` for sm_100a, in the source tree.

``python -m kerrray_b200.build`` compiles each translation unit of ``csrc/`` with nvcc
(``-gencode arch=compute_100a,code=sm_100a``, static CUDA runtime) and links them into one
shared library that exports the C ABI of ``include/kerrray_cuda.h``. The kernel translation
units are compiled with ``-fmad=false``: ``krr_ref.cu`` keeps the reference's rounding of every
product and sum, ``krr_fast.cu`` writes its FMAs explicitly, so no result depends on how the
compiler schedules a particular launch variant.
Rebuilds only when a source or header is newer than the library.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libkerrray_cuda.so"
OBJ = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", str(ROOT / "include"), "--expt-relaxed-constexpr"]
UNITS = {
    "krr_ref.cu": ["-fmad=false"],
    "krr_fast.cu": ["-fmad=false"],
    "krr_abi.cu": [],
    "krr_peak.cu": [],
    "krr_noalloc.cu": [],
    "krr_adjoint.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build libkerrray_cuda.so")


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) +
                  [ROOT / "include" / "kerrray_cuda.h"])


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(src.stat().st_mtime <= t for src in _sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile and link the library if needed; return its path."""
    if not force and up_to_date():
        return LIB
    OBJ.mkdir(exist_ok=True)
    cc = nvcc()
    procs = []
    objs = []
    for unit, extra in UNITS.items():
        obj = OBJ / (Path(unit).stem + ".o")
        objs.append(obj)
        cmd = [cc, *ARCH, *COMMON, *extra, "-c", str(CSRC / unit), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        procs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for unit, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stdout.write(out)
        if p.returncode != 0:
            failed.append(unit)
    if failed:
        raise RuntimeError(f"nvcc failed on {failed}")
    tmp = LIB.with_suffix(".so.tmp")
    link = [cc, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)]
    subprocess.run(link, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
