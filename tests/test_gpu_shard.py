"""The per-rank GPU compute of the sharded extraction, on one GPU: every shard of a 2- and
3-way plan extracted through the C ABI on its SNP slice with rebased block ids and the
whole panel's ploidy, then combined, equals the unsharded extraction bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from steppecu_b200 import shard, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def panel():
    p = synth.generate("c4", seed=7, n_snp=40_000, n_pop=37)
    sel, po = p.selection()
    return p, sel, po


@pytest.mark.parametrize("mode", ["split_f16", "fp32"])
@pytest.mark.parametrize("on_device", [False, True])
def test_shards_equal_unsharded(ctx, panel, mode, on_device):
    import torch

    p, sel, po = panel
    P = len(po) - 1
    rec = p.records_numpy()
    if on_device:
        rec = torch.from_numpy(rec).cuda()
    bid = np.asarray(p.block_id, np.int32)
    whole = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, p.n_block, precision=mode)
    compute = shard.gpu_compute(ctx, rec, p.n_ind, sel, po, precision=mode)
    for G in (2, 3):
        plan = shard.plan_for(bid, p.n_block, G)
        parts = []
        for sh in plan:
            f2 = torch.zeros(P * P * sh.n_block, dtype=torch.float64, device="cuda")
            vp = torch.zeros_like(f2)
            bs = compute(rec[sh.s0:sh.s1], shard.local_block_ids(bid, sh), sh.n_block, f2, vp)
            parts.append((f2.cpu().numpy(), vp.cpu().numpy(), bs))
        got = shard.combine_shards(parts, plan, P, p.n_block)
        assert np.array_equal(got.block_sizes, whole.block_sizes)
        assert np.array_equal(got.vpair, whole.vpair)
        assert np.array_equal(got.f2, whole.f2), f"G={G}: sharded f2 differs from the unsharded extraction"


def test_single_rank_group_assembles_in_place(ctx, panel):
    """extract_blocks_sharded on a one-rank NCCL group: the rank's compute writes straight
    into the full output on the device, which equals the unsharded extraction."""
    import datetime
    import socket

    import torch
    import torch.distributed as dist

    p, sel, po = panel
    P = len(po) - 1
    rec = p.records_numpy()
    bid = np.asarray(p.block_id, np.int32)
    whole = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, p.n_block, precision="split_f16")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        compute = shard.gpu_compute(ctx, rec, p.n_ind, sel, po, precision="split_f16")
        f2, vp, bs = shard.extract_blocks_sharded(compute, rec, bid, p.n_block, P, device="cuda")
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert f2.is_cuda and vp.is_cuda
    assert np.array_equal(bs.cpu().numpy(), whole.block_sizes)
    assert np.array_equal(vp.cpu().numpy(), whole.vpair)
    assert np.array_equal(f2.cpu().numpy(), whole.f2)
