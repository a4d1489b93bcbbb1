"""The ctypes stub that the integration guide gives a KerrRay maintainer: its structures have the ABI's
layout (the package's own bindings of include/kerrray_cuda.h), and on a host without a device
its constructor raises BackendUnavailable, as KerrRay's registry expects (base.py:71-82); the C
example compiles against the header."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from kerrray_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def _stub_source() -> str:
    text = (ROOT / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```python\n(.*?)```", text, flags=re.S)
    src = [b for b in blocks if "class CudaBackend" in b]
    assert len(src) == 1
    return src[0]


def _layout(struct) -> list[tuple[str, int, int]]:
    return [(name, getattr(struct, name).offset, getattr(struct, name).size) for name, _ in struct._fields_]


class BackendUnavailable(RuntimeError):
    """Stands in for kerrray.raytracing.backends.base.BackendUnavailable."""


def _exec_stub() -> dict:
    ns = {"BackendUnavailable": BackendUnavailable, "BatchResult": dict}
    src = _stub_source().replace('"libkerrray_cuda.so"', repr(str(_lib.LIB_PATH)))
    exec(compile(src, "INTEGRATION.md", "exec"), ns)
    return ns


def test_stub_structures_have_the_abi_layout() -> None:
    ns = _exec_stub()
    assert ctypes.sizeof(ns["_Opts"]) == ctypes.sizeof(_lib.KrrOptions)
    assert _layout(ns["_Opts"]) == _layout(_lib.KrrOptions)
    assert ctypes.sizeof(ns["_Res"]) == ctypes.sizeof(_lib.KrrResult)
    assert _layout(ns["_Res"]) == _layout(_lib.KrrResult)


def test_stub_without_a_device_raises_backend_unavailable() -> None:
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    ns = _exec_stub()
    with pytest.raises(BackendUnavailable):
        ns["CudaBackend"]()


def test_c_example_compiles_against_the_header(tmp_path) -> None:
    """The C example (the mixed-precision mask) inside a function that declares its inputs:
    gcc accepts it against include/kerrray_cuda.h with every warning an error."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not found")
    text = (ROOT / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```c\n(.*?)```", text, flags=re.S)
    assert len(blocks) == 1
    src = tmp_path / "example.c"
    src.write_text('#include "kerrray_cuda.h"\n'
                   "int example(const krr_image* images, int32_t n_images, int64_t total_photons, krr_result d_out,\n"
                   "            void* d_ws, void* stream) {\n"
                   "  krr_stats stats;\n" + blocks[0] + "  return (int)stats.critical;\n}\n")
    p = subprocess.run([gcc, "-std=c11", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", str(ROOT / "include"),
                        str(src)], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
