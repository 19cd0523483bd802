"""STPF2BK1 output format pinned against the reference's own f2 directory
(docs/examples/f2_9pop, committed as fixtures by tests/golden/make_golden.py)."""
from __future__ import annotations

import hashlib
import os
from pathlib import Path

import numpy as np
import pytest

from steppecu_b200 import F2Tensor, read_f2, read_f2_dir, write_f2_dir
from steppecu_b200.f2dir import F2DirError, f2_bin_bytes, header_bytes, parse_f2_bin

G = Path(__file__).resolve().parent / "golden"
# The reference checkout, when one is present (STEPPE_REFERENCE_ROOT); the full-file check
# below is skipped without it, the committed fixtures cover the rest.
_REF_ROOT = os.environ.get("STEPPE_REFERENCE_ROOT", "")
REF_EXAMPLE = Path(_REF_ROOT) / "docs" / "examples" / "f2_9pop" if _REF_ROOT else Path("/nonexistent")


@pytest.fixture(scope="module")
def fx():
    return np.load(G / "f2_9pop_head.npz")


def test_header_bytes_match_reference(fx):
    assert header_bytes(int(fx["P"]), int(fx["n_block"])) == (G / "f2_9pop_header.bin").read_bytes()


def test_cache_id_is_sha256_of_f2_bin(fx):
    assert str(fx["meta_f2_cache_id"]) == "sha256:" + str(fx["file_sha256"])
    assert str(fx["meta_pops_sha256"]) == "sha256:" + str(fx["pops_sha256"])


def test_roundtrip_head_blocks(tmp_path, fx):
    P, hb = int(fx["P"]), fx["block_sizes_head"].size
    t = F2Tensor(fx["f2"].copy(), fx["vpair"].copy(), fx["block_sizes_head"].astype(np.int32), P, hb)
    pops = (G / "f2_9pop_pops.txt").read_text().split()
    cid = write_f2_dir(tmp_path / "d", t, pops)
    data = (tmp_path / "d" / "f2.bin").read_bytes()
    assert cid == "sha256:" + hashlib.sha256(data).hexdigest()
    assert (tmp_path / "d" / "pops.txt").read_bytes() == (G / "f2_9pop_pops.txt").read_bytes()
    h = read_f2(tmp_path / "d")
    assert h.P == P and h.n_block == hb and h.pops == pops
    assert np.array_equal(h.to_numpy().ravel(order="F"), fx["f2"])
    assert np.array_equal(h.vpair_to_numpy().ravel(order="F"), fx["vpair"])
    assert h.to_numpy().flags["F_CONTIGUOUS"]


def test_reference_values_are_an_f2_tensor(fx):
    """Structural properties every extract-f2 tensor has: symmetric slabs (the reference's
    GPU output is symmetric to 1e-12, test_f2_blocks_equivalence.cu:149; this file differs
    from exact symmetry by ~3e-17), integer and exactly symmetric vpair, vpair <= block
    size, negative diagonal (-2 mean(h))."""
    P, hb = int(fx["P"]), fx["block_sizes_head"].size
    f2 = fx["f2"].reshape(P, P, hb, order="F")
    vp = fx["vpair"].reshape(P, P, hb, order="F")
    assert np.abs(f2 - f2.transpose(1, 0, 2)).max() <= 1e-12
    assert np.array_equal(vp, vp.transpose(1, 0, 2))
    assert np.array_equal(vp, np.round(vp))
    assert np.all(vp <= fx["block_sizes_head"][None, None, :])
    assert np.all(np.diagonal(f2, axis1=0, axis2=1) < 0)


@pytest.mark.skipif(not (REF_EXAMPLE / "f2.bin").exists(), reason="reference example not present")
def test_full_reference_file_byte_roundtrip(tmp_path, fx):
    data = (REF_EXAMPLE / "f2.bin").read_bytes()
    assert hashlib.sha256(data).hexdigest() == str(fx["file_sha256"])
    t = parse_f2_bin(data)
    assert f2_bin_bytes(t) == data
    t2, pops = read_f2_dir(REF_EXAMPLE)
    assert pops == (G / "f2_9pop_pops.txt").read_text().split()
    assert np.array_equal(t2.block_sizes, fx["block_sizes_all"])


@pytest.mark.parametrize("mutate,msg", [
    (lambda b: b"XXXXXXXX" + b[8:], "bad magic"),
    (lambda b: b[:8] + (2).to_bytes(4, "little") + b[12:], "unsupported version"),
    (lambda b: b[:12] + (2).to_bytes(4, "little") + b[16:], "unsupported dtype"),
    (lambda b: b[:40], "truncated"),
    (lambda b: b[:200], "truncated"),
])
def test_reader_rejects_corrupt_files(tmp_path, fx, mutate, msg):
    P = int(fx["P"])
    t = F2Tensor(fx["f2"][: P * P].copy(), fx["vpair"][: P * P].copy(), fx["block_sizes_head"][:1].astype(np.int32), P, 1)
    d = tmp_path / "bad"
    write_f2_dir(d, t, (G / "f2_9pop_pops.txt").read_text().split())
    (d / "f2.bin").write_bytes(mutate((d / "f2.bin").read_bytes()))
    with pytest.raises(F2DirError, match=msg):
        read_f2_dir(d)


def test_writer_rejects_degenerate(tmp_path):
    with pytest.raises(F2DirError):
        write_f2_dir(tmp_path / "x", F2Tensor(np.zeros(0), np.zeros(0), np.zeros(0, np.int32), 0, 0), [])
    with pytest.raises(F2DirError):
        write_f2_dir(tmp_path / "y", F2Tensor(np.zeros(4), np.zeros(4), np.zeros(1, np.int32), 2, 1), ["a"])
