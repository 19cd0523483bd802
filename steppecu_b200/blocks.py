"""Jackknife block assignment: the AT2 block walk of core::assign_blocks
(src/core/domain/block_partition_rule.cpp:18-85 in the reference).

A new block starts at the first SNP, whenever the chromosome changes, and whenever
(pos - anchor) >= width, where the anchor is the position of the block's first SNP. The
comparison is evaluated exactly as written (a difference, then >=), so floating-point
knife edges fall the same way as in the reference. With an all-zero genetic map and a
non-zero physical axis, the walk runs on physical positions with a 2 Mb window.
"""
from __future__ import annotations

import numpy as np

BP_FALLBACK_WINDOW = 2.0e6  # include/steppe/config.hpp:55 (kBpFallbackWindow)


def _walk(chrom: np.ndarray, pos: np.ndarray, window: float) -> tuple[np.ndarray, int]:
    M = pos.size
    block_id = np.empty(M, dtype=np.int32)
    # Chromosome runs (a change of chromosome always opens a block).
    change = np.flatnonzero(np.diff(chrom)) + 1
    starts = np.concatenate([[0], change])
    ends = np.concatenate([change, [M]])
    b = 0
    for s0, s1 in zip(starts.tolist(), ends.tolist()):
        seg = pos[s0:s1]
        j = 0
        n = s1 - s0
        while j < n:
            anchor = seg[j]
            # Candidate cut from a sorted search, then settle it with the exact predicate.
            k = j + 1 + int(np.searchsorted(seg[j + 1:], anchor + window, side="left"))
            k = min(max(k, j + 1), n)
            while k > j + 1 and (seg[k - 1] - anchor) >= window:
                k -= 1
            while k < n and not ((seg[k] - anchor) >= window):
                k += 1
            block_id[s0 + j:s0 + k] = b
            b += 1
            j = k
    return block_id, b


def assign_blocks(chrom, genpos_morgans, block_size_morgans: float = 0.05, physpos=None,
                  bp_window: float = BP_FALLBACK_WINDOW) -> tuple[np.ndarray, int]:
    """Returns (block_id int32 [M], n_block). An illegal width (<= 0 or NaN) or M == 0
    gives an empty partition, as in the reference."""
    chrom = np.asarray(chrom, dtype=np.int64)
    gp = np.asarray(genpos_morgans, dtype=np.float64)
    M = min(chrom.size, gp.size)
    if not (block_size_morgans > 0.0) or M <= 0:
        return np.zeros(0, np.int32), 0
    chrom, gp = chrom[:M], gp[:M]
    if physpos is not None and bp_window > 0.0:
        pp = np.asarray(physpos, dtype=np.float64)
        if pp.size >= M and not np.any(gp != 0.0) and np.any(pp[:M] != 0.0):
            return _walk(chrom, pp[:M], bp_window)
    return _walk(chrom, gp, block_size_morgans)


def block_ranges(block_id: np.ndarray, n_block: int) -> list[tuple[int, int]]:
    """Inverse of assign_blocks (block_partition_rule.hpp:56-96): [begin, end) per block.
    Raises ValueError for an out-of-range or decreasing id."""
    block_id = np.asarray(block_id)
    if block_id.size == 0 or n_block <= 0:
        return []
    if block_id.min() < 0 or block_id.max() >= n_block:
        raise ValueError("block_id out of range")
    if np.any(np.diff(block_id) < 0):
        raise ValueError("block_id is not non-decreasing; the partition is not contiguous")
    out = [(0, 0)] * n_block
    edges = np.flatnonzero(np.diff(block_id)) + 1
    starts = np.concatenate([[0], edges])
    ends = np.concatenate([edges, [block_id.size]])
    for s0, s1 in zip(starts.tolist(), ends.tolist()):
        out[int(block_id[s0])] = (s0, s1)
    return out
