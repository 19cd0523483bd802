"""The one-shot extraction's plan cache (stpf2_abi.cu, PlanCache): a repeated host-buffer
extraction with an identical request reuses the plan built for the first call. The key is
the request's content, not its pointers, and never the records: a changed array at the
same address, or other records under the same request, must give what a fresh context
gives, bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import steppecu_b200 as sb
from steppecu_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def panel():
    return synth.generate("c2", seed=5, n_snp=20_000, n_pop=130)  # two row tiles


def _fresh(rec, p, sel, po, bid, nb, **kw):
    with sb.Context(0) as c:
        return c.extract_blocks(rec, p.n_ind, sel, po, bid, nb, **kw)


def _same(a, b):
    return np.array_equal(a.f2, b.f2) and np.array_equal(a.vpair, b.vpair) and np.array_equal(a.block_sizes, b.block_sizes)


@pytest.mark.parametrize("mode", ["fixed_i8", "split_f16"])
def test_repeated_request_reuses_plan(ctx, panel, mode):
    p = panel
    sel, po = p.selection()
    rec = p.records_numpy()
    assert p.n_block >= 2  # the segmented host-output path
    first = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    again = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    assert _same(first, again)
    # Other records under the same request: re-detected ploidy, re-decoded.
    rec2 = np.ascontiguousarray(rec[::-1])
    got = ctx.extract_blocks(rec2, p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    assert _same(got, _fresh(rec2, p, sel, po, p.block_id, p.n_block, precision=mode))


def test_changed_arrays_at_the_same_address_rebuild(ctx, panel):
    p = panel
    sel, po = p.selection()
    rec = p.records_numpy()
    bid = p.block_id.copy()
    ctx.extract_blocks(rec, p.n_ind, sel, po, bid, p.n_block, precision="fixed_i8")
    bid[bid == 1] = 0  # block 1 joins block 0 (and becomes empty), same buffer
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, p.n_block, precision="fixed_i8")
    assert got.block_sizes[1] == 0
    assert _same(got, _fresh(rec, p, sel, po, bid, p.n_block, precision="fixed_i8"))
    # A changed selection at the same address: the first two samples swap populations'
    # order within the selection (same counts, other samples).
    sel2 = sel.copy()
    sel2[[0, -1]] = sel2[[-1, 0]]
    got = ctx.extract_blocks(rec, p.n_ind, sel2, po, bid, p.n_block, precision="fixed_i8")
    assert _same(got, _fresh(rec, p, sel2, po, bid, p.n_block, precision="fixed_i8"))
    # A different precision is a different plan.
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, p.n_block, precision="split_f16")
    assert _same(got, _fresh(rec, p, sel, po, bid, p.n_block, precision="split_f16"))


def test_cached_plan_survives_another_plan_in_its_workspace(ctx, panel):
    """A streamed extraction of another request builds its plan in the same operand-plane
    workspace (other block padding, other populations); the next repeat of the cached request
    must rebuild rather than read stale padding columns: equal to a fresh context, bit for bit."""
    p = panel
    sel, po = p.selection()
    rec = p.records_numpy()
    want = _fresh(rec, p, sel, po, p.block_id, p.n_block, precision="fixed_i8")
    ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8")  # cached
    sel2, po2 = p.selection(list(range(0, p.n_pop, 2)))
    bid2 = (np.arange(p.n_snp) // 777).astype(np.int32)  # other padding
    ctx.extract_streamed(rec, p.n_ind, sel2, po2, bid2, int(bid2[-1]) + 1, lambda *a: None, precision="fixed_i8")
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8")
    assert _same(got, want)
