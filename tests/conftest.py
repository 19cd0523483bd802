"""Shared test setup: the `gpu` marker, import paths, and on-demand native builds."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through libstpf2.so")


def pytest_sessionstart(session):
    # Build the oracle (and libstpf2.so) if they are missing; both are in-tree outputs.
    from steppecu_b200 import build

    if not (ROOT / "oracle" / "liboracle.so").exists():
        build.build_oracle()
    if not build.LIB.exists():
        build.build_lib()


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def ctx():
    from steppecu_b200 import Context

    c = Context(0)
    yield c
    c.close()
