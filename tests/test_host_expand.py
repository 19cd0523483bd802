"""The host side of the host-output transfer (steppecu_b200/csrc/host_expand.cpp), on CPU: it
is plain C++, so it is compiled here with tests/native/expand_check.cpp. It packs random
symmetric count slabs in the device packer's order and checks the widened slabs, and fills
the lower tiles of symmetric FP64 slabs from their upper tiles, bit for bit, for P from 1 to
1,001, 16- and 32-bit counts, on 32-byte aligned slabs (the AVX2 paths where the CPU has
AVX2) and misaligned ones (the element paths)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_expand_and_mirror_fill_both_halves_exactly(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "expand_check"
    subprocess.run([gxx, "-O2", "-std=c++17", str(ROOT / "tests" / "native" / "expand_check.cpp"),
                    str(ROOT / "steppecu_b200" / "csrc" / "host_expand.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
