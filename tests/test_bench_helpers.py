"""The bench line's arithmetic, on CPU: the metric's units, the issued tensor work of the
split contraction counted from its MMA schedule, and the bytes the host-output extraction
downloads (upper tiles: f2 in FP64, vpair as packed counts)."""
from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
_spec = importlib.util.spec_from_file_location("bench_module", ROOT / "bench.py")
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_units_count_unordered_pairs():
    assert bench.units(1000, 1_150_000) == 1_150_000 * 1000 * 999 / 2
    assert bench.units(1, 10) == 0


@pytest.mark.parametrize("P", [100, 128, 129, 1000])
def test_issued_work_matches_mma_count(P):
    sizes = np.array([1, 31, 32, 33, 1600, 0, 6000])
    bid = np.repeat(np.arange(sizes.size), sizes)
    w = bench.issued_tensor_work(P, bid, sizes.size, con_ms=1.0, peak=1000.0)
    rt = -(-P // 128)
    pairs = rt * (rt + 1) // 2
    stages = sum(-(-int(k) // 32) for k in sizes)
    # per stage of a tile pair: 14 f16 MMAs of 128x128x16 and one i8 MMA of 128x128x32
    assert w["f16_flops"] == pairs * stages * 14 * 2 * 128 * 128 * 16
    assert w["i8_ops"] == pairs * stages * 2 * 128 * 128 * 32
    assert w["f16_tflops"] == pytest.approx(w["f16_flops"] / 1e-3 / 1e12)


@pytest.mark.parametrize("P", [1, 5, 128, 129, 300, 1000])
def test_host_d2h_bytes_match_the_copies(P):
    B = 3
    upper = np.zeros((P, P), bool)  # [row i, column j]: the packed upper tiles
    for r0 in range(0, P, 128):
        upper[r0:r0 + 128, r0:P] = True
    assert np.all(upper | upper.T)  # the tiles and their transposes cover every element
    t = -(-P // 128)
    packed = t * (t + 1) // 2 * 128 * 128  # counts per slab, with each tile padded to 128 x 128
    assert packed >= int(upper.sum())
    assert bench.host_d2h_bytes(P, B) == B * (8 * int(upper.sum()) + 2 * packed)
    assert bench.host_d2h_bytes(P, B, wide=True) == B * (8 * int(upper.sum()) + 4 * packed)
