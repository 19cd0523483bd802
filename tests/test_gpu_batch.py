"""Grouped batches (stp_f2_extract_batch) against one-request extraction and the oracle.

Each request of a batch selects its own populations and has its own block map over one
shared panel. The grouped path (union transpose, per-request decode from shared canonical
genotypes, one contraction launch over all requests) must reproduce the one-request path
bit for bit: same centres, same tiles, same MMA order per block.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from steppecu_b200 import F2Tensor, synth

pytestmark = pytest.mark.gpu


def random_blocks(rng, n_snp: int, mean: float) -> tuple[np.ndarray, int]:
    """A contiguous partition with sizes ~ exponential(mean), 1-SNP blocks included."""
    sizes = []
    left = n_snp
    while left > 0:
        k = int(min(left, max(1, rng.exponential(mean))))
        sizes.append(k)
        left -= k
    bid = np.repeat(np.arange(len(sizes), dtype=np.int32), sizes)
    return bid, len(sizes)


@pytest.fixture(scope="module")
def panel():
    return synth.generate("c4", seed=11, n_snp=20_000, n_pop=140)


def make_requests(panel, seed: int, sizes):
    rng = np.random.default_rng(seed)
    reqs = []
    for i, P in enumerate(sizes):
        pops = np.sort(rng.choice(panel.n_pop, size=P, replace=False)).tolist()
        sel, po = panel.selection(pops)
        bid, nb = random_blocks(rng, panel.n_snp, mean=[300.0, 900.0, 40.0][i % 3])
        reqs.append({"sel_rows": sel, "pop_offsets": po, "block_id": bid, "n_block": nb})
    return reqs


@pytest.mark.parametrize("precision", ["split_f16", "split_bf16", "split_f16_fine"])
def test_batch_equals_one_request_extraction(ctx, panel, precision):
    reqs = make_requests(panel, 3, [1, 4, 9, 140, 23, 2, 130])
    reqs[2]["ploidy"] = "diploid"
    reqs[4]["sample_ploidy"] = np.where(np.arange(reqs[4]["sel_rows"].size) % 3 == 0, 1, 2).astype(np.int32)
    rec = panel.records_numpy()
    got = ctx.extract_batch(rec, panel.n_ind, reqs, precision=precision)
    ms = ctx.last_batch_times(len(reqs))
    for q, t in zip(reqs, got):
        one = ctx.extract_blocks(rec, panel.n_ind, q["sel_rows"], q["pop_offsets"], q["block_id"], q["n_block"],
                                 precision=precision, sample_ploidy=q.get("sample_ploidy"),
                                 ploidy=q.get("ploidy", "auto"))
        assert np.array_equal(t.block_sizes, one.block_sizes)
        assert np.array_equal(t.vpair, one.vpair)
        assert np.array_equal(t.f2, one.f2)
    assert np.all(np.isfinite(ms)) and np.all(ms > 0)


def test_batch_against_oracle(ctx, panel):
    reqs = make_requests(panel, 5, [5, 37])
    rec = panel.records_numpy()
    got = ctx.extract_batch(rec, panel.n_ind, reqs, precision="split_f16")
    for q, t in zip(reqs, got):
        pl = oracle.detect_ploidy_pa(rec, q["sel_rows"])
        f2, vp, bs = oracle.f2_from_panel(rec, q["sel_rows"], q["pop_offsets"], q["block_id"], q["n_block"], pl, threads=8)
        want = F2Tensor(f2, vp, bs, len(q["pop_offsets"]) - 1, q["n_block"])
        assert np.array_equal(t.block_sizes, want.block_sizes)
        assert np.array_equal(t.vpair, want.vpair)
        bad = np.abs(t.f2 - want.f2) > 2e-7 + 5e-6 * np.abs(want.f2)
        assert not bad.any(), int(bad.sum())


def test_mixed_batch_device_records_and_fp32(ctx, panel):
    """Device-resident records and device outputs; an FP32 request runs on its own (NaN
    completion time) beside the grouped tensor-core requests."""
    import torch

    reqs = make_requests(panel, 7, [12, 3, 60])
    rec_h = panel.records_numpy()
    rec_d = torch.from_numpy(rec_h).cuda()
    outs = []
    for q in reqs:
        n = (len(q["pop_offsets"]) - 1) ** 2 * q["n_block"]
        outs.append((torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.float64, device="cuda")))
    got = ctx.extract_batch(rec_d, panel.n_ind, reqs, precision="split_f16", out=outs)
    for q, (f2, vp, bs) in zip(reqs, got):
        one = ctx.extract_blocks(rec_h, panel.n_ind, q["sel_rows"], q["pop_offsets"], q["block_id"], q["n_block"],
                                 precision="split_f16")
        assert np.array_equal(bs, one.block_sizes)
        assert np.array_equal(vp.cpu().numpy(), one.vpair)
        assert np.array_equal(f2.cpu().numpy(), one.f2)
    # FP32 requests are not grouped.
    ctx.extract_batch(rec_h, panel.n_ind, reqs[:2], precision="fp32")
    assert np.all(np.isnan(ctx.last_batch_times(2)))
