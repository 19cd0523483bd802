"""The host-side fill of the band download (steppecu_b200/csrc/host_mirror.cpp), on CPU: it is
plain C++, so it is compiled here with tests/native/mirror_check.cpp, which checks every
slab it fills against the full symmetric slab bit for bit, for P from 1 to 1,001, on 32-byte
aligned slabs (the AVX2 path where the CPU has AVX2) and misaligned ones (the scalar path)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_mirror_fills_lower_tiles_exactly(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "mirror_check"
    subprocess.run([gxx, "-O2", "-std=c++17", str(ROOT / "tests" / "native" / "mirror_check.cpp"),
                    str(ROOT / "steppecu_b200" / "csrc" / "host_mirror.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
