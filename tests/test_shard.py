"""Block sharding for N > 1 GPUs, on CPU: the shard planner against the reference's own
planner cases, the combine's guards, and world-size 2 and 3 gloo runs of the sharded
extraction whose assembled tensor must equal the whole-panel oracle bit for bit."""
from __future__ import annotations

import multiprocessing as mp
import socket

import numpy as np
import pytest

import oracle
import shard_worker
from steppecu_b200.shard import Shard, block_ranges, combine_shards, plan_block_shards, plan_for


def ranges_from_sizes(sizes):
    out, c = [], 0
    for s in sizes:
        out.append((c, c + s))
        c += s
    return out


# The expected plans of the reference's planner tests (tests/unit/test_shard_plan.cpp:176-228),
# as (block sizes, G, [(b0, b1, s0, s1), ...]).
PLAN_CASES = [
    ([10] * 6, 3, [(0, 2, 0, 20), (2, 4, 20, 40), (4, 6, 40, 60)]),
    ([10] * 4, 1, [(0, 4, 0, 40)]),
    ([], 3, [(0, 0, 0, 0)] * 3),
    ([10, 10, 10], 5, [(0, 1, 0, 10), (1, 2, 10, 20), (2, 3, 20, 30), (0, 0, 0, 0), (0, 0, 0, 0)]),
    ([0, 0, 0, 0], 3, [(0, 1, 0, 0), (1, 2, 0, 0), (2, 4, 0, 0)]),
    ([1000, 1, 1], 3, [(0, 1, 0, 1000), (1, 3, 1000, 1002), (0, 0, 0, 0)]),
    ([1, 1, 1, 1, 1000], 3, [(0, 5, 0, 1004), (0, 0, 0, 0), (0, 0, 0, 0)]),
    ([5] * 5, 2, [(0, 3, 0, 15), (3, 5, 15, 25)]),
]


@pytest.mark.parametrize("sizes,G,want", PLAN_CASES)
def test_plan_matches_reference_cases(sizes, G, want):
    plan = plan_block_shards(ranges_from_sizes(sizes), G)
    assert [(s.b0, s.b1, s.s0, s.s1) for s in plan] == want


def test_plan_zero_devices_is_an_error():
    with pytest.raises(ValueError):
        plan_block_shards(ranges_from_sizes([10, 10]), 0)


@pytest.mark.parametrize("G", [1, 2, 3, 4, 7, 8, 16])
def test_plan_structure_on_mixed_sizes(G):
    """Contiguous, block-aligned, covering, and empty shards only at the end
    (test_shard_plan.cpp:68-118's structure check), on lognormal block sizes."""
    rng = np.random.default_rng(G)
    sizes = np.maximum(1, np.round(np.exp(rng.normal(6.0, 0.8, size=37)))).astype(int).tolist()
    ranges = ranges_from_sizes(sizes)
    plan = plan_block_shards(ranges, G)
    assert len(plan) == G
    nb, s, seen_empty = 0, 0, False
    for sh in plan:
        if sh.empty():
            seen_empty = True
            continue
        assert not seen_empty
        assert (sh.b0, sh.s0) == (nb, s)
        assert sh.s0 == ranges[sh.b0][0] and sh.s1 == ranges[sh.b1 - 1][1]
        nb, s = sh.b1, sh.s1
    assert nb == len(sizes)
    target = -(-sum(sizes) // G)
    filled = [sh for sh in plan if not sh.empty()]
    for sh in filled[:-1]:  # every shard closed before the last one reached the target
        assert sum(sizes[sh.b0:sh.b1]) >= target


def test_block_ranges_rules():
    assert block_ranges(np.array([0, 0, 1, 1, 1, 3]), 4) == [(0, 2), (2, 5), (0, 0), (5, 6)]
    assert block_ranges(np.zeros(0, np.int32), 3) == []
    with pytest.raises(ValueError, match="out of range"):
        block_ranges(np.array([0, 4]), 4)
    with pytest.raises(ValueError, match="non-decreasing"):
        block_ranges(np.array([0, 1, 0]), 2)


def test_combine_guards():
    P = 2
    sh = [Shard(0, 2, 0, 10), Shard(2, 3, 10, 15)]
    ok = [(np.ones(8), np.ones(8), np.ones(2, np.int32)), (np.ones(4), np.ones(4), np.ones(1, np.int32))]
    t = combine_shards(ok, sh, P, 3)
    assert t.f2.size == 12 and np.array_equal(t.block_sizes, [1, 1, 1])
    with pytest.raises(ValueError, match="partials count"):
        combine_shards(ok[:1], sh, P, 3)
    with pytest.raises(ValueError, match="storage size"):
        combine_shards([ok[0], (np.ones(3), np.ones(4), np.ones(1, np.int32))], sh, P, 3)
    with pytest.raises(ValueError, match="cover"):
        combine_shards(ok, sh, P, 4)


def test_combine_of_oracle_shards_equals_whole_panel():
    """Single-process form of the fan-out: per-shard oracle extractions on rebased block ids,
    combined, equal the whole-panel extraction bit for bit."""
    rec, sel, po, bid, nb, P, pl = shard_worker.panel_case("panel")
    want = oracle.f2_from_panel(rec, sel, po, bid, nb, pl)
    for G in (2, 3, 5):
        plan = plan_for(bid, nb, G)
        parts = []
        for sh in plan:
            if sh.empty():
                parts.append((np.zeros(0), np.zeros(0), np.zeros(0, np.int32)))
                continue
            lbid = (bid[sh.s0:sh.s1] - sh.b0).astype(np.int32)
            parts.append(oracle.f2_from_panel(rec[sh.s0:sh.s1], sel, po, lbid, sh.n_block, pl))
        got = combine_shards(parts, plan, P, nb)
        for a, b in zip((got.f2, got.vpair, got.block_sizes), want):
            assert np.array_equal(a, b)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(world: int, case: str, out_dir, fail_rank: int = -1):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=shard_worker.run, args=(r, world, port, case, str(out_dir), fail_rank))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
        p.join()
    crashes = {f.name: f.read_text() for f in out_dir.glob("crash*.txt")}
    assert not alive, "a rank did not finish"
    assert not crashes, crashes
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


@pytest.mark.parametrize("world,case", [(2, "panel"), (3, "panel"), (3, "two_blocks")])
def test_gloo_sharded_extraction_equals_whole_panel(tmp_path, world, case):
    _run_ranks(world, case, tmp_path)
    rec, sel, po, bid, nb, P, pl = shard_worker.panel_case(case)
    want_f2, want_vp, want_bs = oracle.f2_from_panel(rec, sel, po, bid, nb, pl)
    got = np.load(tmp_path / "got.npz")
    assert np.array_equal(got["f2"], want_f2)
    assert np.array_equal(got["vpair"], want_vp)
    assert np.array_equal(got["block_sizes"], want_bs)
    plan = plan_for(bid, nb, world)
    for r, sh in enumerate(plan):
        seen = np.load(tmp_path / f"seen{r}.npy")
        if sh.empty():
            assert seen.shape[0] == 0  # an empty shard computes nothing
        else:  # each rank saw its SNP slice and dense zero-based local block ids
            assert seen.tolist() == [[sh.s1 - sh.s0, sh.n_block, 0, sh.n_block - 1]]


def test_gloo_failed_rank_fails_every_rank(tmp_path):
    """A rank whose compute raises: every rank raises instead of waiting in the exchange."""
    _run_ranks(2, "panel", tmp_path, fail_rank=1)
    e0 = (tmp_path / "error0.txt").read_text()
    e1 = (tmp_path / "error1.txt").read_text()
    assert "another rank failed" in e0
    assert "rank 1 failed" in e1
    assert not (tmp_path / "got.npz").exists()
