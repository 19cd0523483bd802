"""The reference-side adapter (steppecu_b200/adapter/b200_backend.cpp) compiles against the
reference's own headers.

The adapter (`B200Backend : ComputeBackend`) is the drop-in a maintainer adds on the
reference side. Compiling it with `override` on every forwarded virtual checks that each
signature matches the reference's ComputeBackend (compute_f2 / compute_f2_blocks /
_device / _into / _streamed, decode_af, decode_af_compact_filter,
detect_sample_ploidy_device) and that the reference types it fills (DeviceF2Blocks,
DeviceDecodeResult, StreamTarget's host and disk tiers, F2DiskHeader) have the members it
uses. It runs wherever the reference sources are present (the checkout oracle/Makefile
builds from); elsewhere it is skipped.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
ADAPTER = ROOT / "steppecu_b200" / "adapter" / "b200_backend.cpp"


def reference_root() -> Path | None:
    try:
        out = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "print-ref"], capture_output=True, text=True,
                             check=True).stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return None
    ref = Path(out) if out else None
    return ref if ref and (ref / "src" / "device" / "backend.hpp").exists() else None


def test_adapter_compiles_against_reference_headers():
    ref = reference_root()
    if ref is None or shutil.which("g++") is None:
        pytest.skip("reference sources or g++ not available")
    cuda_inc = Path("/usr/local/cuda/include")
    # The reference's check.cuh names four cuFFT statuses that only CUDA 13 headers declare;
    # distinct stand-in values let it parse against older headers.
    shims = [f"-D{name}={1000 + k}" for k, name in enumerate(
        ["CUFFT_MISSING_DEPENDENCY", "CUFFT_NVRTC_FAILURE", "CUFFT_NVJITLINK_FAILURE", "CUFFT_NVSHMEM_FAILURE"])]
    cmd = ["g++", "-std=c++20", "-fsyntax-only", "-Wall", f"-I{ref / 'src'}", f"-I{ref / 'include'}",
           f"-I{ROOT / 'include'}", f"-I{cuda_inc}", *shims, str(ADAPTER)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_adapter_binds_every_hot_path_virtual():
    src = ADAPTER.read_text()
    for name in ("compute_f2(", "compute_f2_blocks(", "compute_f2_blocks_device(", "compute_f2_blocks_into(",
                 "compute_f2_blocks_streamed(", "decode_af(", "decode_af_compact_filter(",
                 "detect_sample_ploidy_device("):
        assert name in src, name
