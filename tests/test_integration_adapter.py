"""The C++ adapter in INTEGRATION.md compiles against the reference's own headers.

The adapter (`B200Backend : ComputeBackend`) is the drop-in a maintainer adds on the
reference side. Compiling it with `override` on every forwarded virtual checks that each
signature matches the reference's ComputeBackend and that every pure virtual is
implemented. It runs wherever the reference sources are present (the path the oracle's
Makefile builds from); elsewhere it is skipped.
"""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def reference_root() -> Path | None:
    m = re.search(r"^REF \?= (.+)$", (ROOT / "oracle" / "Makefile").read_text(), re.M)
    ref = Path(m.group(1).strip()) if m else None
    return ref if ref and (ref / "src" / "device" / "backend.hpp").exists() else None


def test_adapter_compiles_against_reference_headers(tmp_path):
    ref = reference_root()
    if ref is None or shutil.which("g++") is None:
        pytest.skip("reference sources or g++ not available")
    blocks = re.findall(r"```cpp\n(.*?)```", (ROOT / "INTEGRATION.md").read_text(), re.S)
    assert blocks, "INTEGRATION.md has no C++ adapter"
    src = tmp_path / "b200_backend.cpp"
    src.write_text(blocks[0])
    cuda_inc = Path("/usr/local/cuda/include")
    # The reference's check.cuh names four cuFFT statuses that only CUDA 13 headers declare;
    # distinct stand-in values let it parse against older headers.
    shims = [f"-D{name}={1000 + k}" for k, name in enumerate(
        ["CUFFT_MISSING_DEPENDENCY", "CUFFT_NVRTC_FAILURE", "CUFFT_NVJITLINK_FAILURE", "CUFFT_NVSHMEM_FAILURE"])]
    cmd = ["g++", "-std=c++20", "-fsyntax-only", f"-I{ref / 'src'}", f"-I{ref / 'include'}", f"-I{ROOT / 'include'}",
           f"-I{cuda_inc}", *shims, str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
