"""The C-ABI library: it loads, exports every symbol include/stpf2.h declares, and fails loudly (no CPU fallback) when there is no GPU."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from steppecu_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "stpf2.h"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(stp_[a-z0-9_]+)\s*\(", text))


def test_header_declarations_have_bindings():
    decl = declared_functions()
    assert decl, "no declarations parsed"
    assert decl == set(_lib.SIGNATURES), decl ^ set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (stp_[a-z0-9_]+)$", out, flags=re.M))
    missing = declared_functions() - exported
    assert not missing, missing


def test_library_loads_and_reports_abi_version():
    L = _lib.lib()
    assert L.stp_abi_version() == 2


def test_no_device_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    st = C.c_int(0)
    h = _lib.lib().stp_create(0, C.byref(st))
    assert not h and st.value == _lib.STP_NO_DEVICE
    assert b"CUDA" in _lib.lib().stp_last_error()
