"""The committed tile-class table (steppecu_b200/tile_classes.json, written by
steppecu_b200/autotune.py on a B200) is well formed, and the library's built-in default is
the same mask, so a caller that never loads the table (the C++ adapter) gets the measured
choice too."""
from __future__ import annotations

import json
import re
from pathlib import Path

from steppecu_b200 import autotune

ROOT = Path(__file__).resolve().parents[1]


def test_table_is_well_formed_and_matches_the_builtin_default():
    t = json.loads(autotune.TABLE.read_text())
    assert len(t["classes"]) == autotune.N_CLASSES
    mask = autotune.load_mask()
    assert mask == sum(1 << c["class"] for c in t["classes"] if c["partial"])
    assert all(c["partial"] == (c["partial_ms"] < c["full_ms"]) for c in t["classes"])
    hdr = (ROOT / "steppecu_b200" / "csrc" / "stpf2_internal.cuh").read_text()
    m = re.search(r"kDefaultPartialFeed = (0x[0-9A-Fa-f]+)u", hdr)
    assert m and int(m.group(1), 16) == mask
