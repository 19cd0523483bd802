"""Block-sharded extraction over several GPUs (one process per GPU).

Jackknife blocks are independent, so a request splits into contiguous runs of whole blocks,
one per rank. Each rank decodes and contracts its own run of SNPs on its own GPU; the data
path has no collective. The one exchange is the assembly of the result: every rank sends its
f2 / vpair / block_sizes slab to rank 0, which receives it in place at the slab's block
offset (point-to-point, NCCL over NVLink on GPUs, gloo on CPU).

`plan_block_shards` restates the reference's shard planner (src/device/shard_plan.cpp:17-70):
contiguous runs of blocks, each closed once it holds at least ceil(total SNPs / G) SNPs,
while more devices and blocks remain; ranks past the last run get empty shards.
`block_ranges` restates core::block_ranges (src/core/domain/block_partition_rule.hpp:56-96),
`validate_partials` the combine's precondition guard
(src/core/fstats/f2_partials_validate.hpp:25-100) and `combine_shards` the host-staged
combine (src/core/fstats/f2_combine.cpp:21-56).

Ploidy: the reference decodes the whole panel before it shards (ploidy from the panel's
first min(1000, M) SNPs), so a rank whose shard starts later must not detect ploidy on its
own SNPs. `gpu_compute` detects it once on the whole panel and passes it to every shard,
which makes the sharded result bit-identical to the unsharded one.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from .f2dir import F2Tensor


@dataclass(frozen=True)
class Shard:
    """DeviceShard (src/device/shard_plan.hpp): blocks [b0, b1), SNP columns [s0, s1)."""
    b0: int = 0
    b1: int = 0
    s0: int = 0
    s1: int = 0

    @property
    def n_block(self) -> int:
        return self.b1 - self.b0

    def empty(self) -> bool:
        return self.b1 <= self.b0


def block_ranges(block_id, n_block: int) -> list[tuple[int, int]]:
    """[begin, end) SNP range of every block of a contiguous non-decreasing partition. A
    block with no SNPs keeps the empty range (0, 0), as in the reference. Raises ValueError on
    an id outside [0, n_block) or a decreasing id."""
    bid = np.asarray(block_id, dtype=np.int64).reshape(-1)
    M = bid.size
    if M == 0 or n_block <= 0:
        return []
    if bid.min() < 0 or bid.max() >= n_block:
        s = int(np.flatnonzero((bid < 0) | (bid >= n_block))[0])
        raise ValueError(f"block_ranges: block_id[{s}] = {int(bid[s])} is out of range [0, {n_block})")
    dec = np.flatnonzero(np.diff(bid) < 0)
    if dec.size:
        s = int(dec[0]) + 1
        raise ValueError(f"block_ranges: block_id is not non-decreasing at column {s}; the partition "
                         "is not contiguous")
    ranges = [(0, 0)] * n_block
    edges = np.flatnonzero(np.diff(bid)) + 1
    starts = np.concatenate([[0], edges])
    ends = np.concatenate([edges, [M]])
    for s, e in zip(starts.tolist(), ends.tolist()):
        ranges[int(bid[s])] = (s, e)
    return ranges


def plan_block_shards(ranges: Sequence[tuple[int, int]], G: int) -> list[Shard]:
    """G contiguous block runs balanced by SNP count (shard_plan.cpp:17-70)."""
    if G <= 0:
        raise ValueError("plan_block_shards: G == 0 (at least one device is needed)")
    n = len(ranges)
    plan = [Shard()] * G
    if n == 0:
        return plan
    total = sum(e - s for s, e in ranges)
    target = -(-total // G)
    g, b0, acc = 0, 0, 0
    for b in range(n):
        acc += ranges[b][1] - ranges[b][0]
        if g + 1 < G and acc >= target and b + 1 < n:
            plan[g] = Shard(b0, b + 1, ranges[b0][0], ranges[b][1])
            g, b0, acc = g + 1, b + 1, 0
    plan[g] = Shard(b0, n, ranges[b0][0], ranges[n - 1][1])
    return plan


def plan_for(block_id, n_block: int, G: int) -> list[Shard]:
    """plan_multigpu_shards (src/core/fstats/f2_blocks_multigpu_core.cpp:88-97)."""
    return plan_block_shards(block_ranges(block_id, n_block), G)


def local_block_ids(block_id, sh: Shard) -> np.ndarray:
    """The shard's zero-based block ids (block_id[s0 + k] - b0), as the fan-out hands them to
    each device (f2_blocks_multigpu_core.cpp:63-67)."""
    return (np.asarray(block_id[sh.s0:sh.s1], dtype=np.int64) - sh.b0).astype(np.int32)


def validate_partials(parts: Sequence[tuple[np.ndarray, np.ndarray, np.ndarray]], shards: Sequence[Shard],
                      P: int, n_block: int) -> None:
    """The combine's precondition guard (f2_partials_validate.hpp:25-100): one partial per
    shard, each with P*P*span f2/vpair values and span block sizes, and the shards' spans
    adding up to n_block."""
    if len(parts) != len(shards):
        raise ValueError(f"partials count ({len(parts)}) != shards count ({len(shards)})")
    if P < 0 or n_block < 0:
        raise ValueError("negative P or n_block_full")
    covered = 0
    for g, ((f2, vp, bs), sh) in enumerate(zip(parts, shards)):
        span = sh.b1 - sh.b0
        if span > 0:
            want = P * P * span
            if np.size(f2) != want or np.size(vp) != want or np.size(bs) != span:
                raise ValueError(f"partial[{g}] storage size mismatch: expected f2/vpair={want} "
                                 f"(P*P*n_block), block_sizes={span}; got f2={np.size(f2)}, "
                                 f"vpair={np.size(vp)}, block_sizes={np.size(bs)}")
        covered += span
    if covered != n_block:
        raise ValueError(f"shards cover {covered} blocks but n_block_full = {n_block} "
                         "(the shards must tile [0, n_block_full))")


def combine_shards(parts: Sequence[tuple[np.ndarray, np.ndarray, np.ndarray]], shards: Sequence[Shard],
                   P: int, n_block: int) -> F2Tensor:
    """The full F2BlockTensor from per-shard (f2, vpair, block_sizes) partials, each copied
    into place at its block offset (f2_combine.cpp:21-56). Shards are disjoint, so every slab
    is written once and the result equals the unsharded one bit for bit."""
    validate_partials(parts, shards, P, n_block)
    slab = P * P
    f2 = np.zeros(slab * n_block)
    vp = np.zeros(slab * n_block)
    bs = np.zeros(n_block, np.int32)
    for (pf2, pvp, pbs), sh in zip(parts, shards):
        if sh.empty():
            continue
        f2[slab * sh.b0:slab * sh.b1] = np.asarray(pf2).reshape(-1)
        vp[slab * sh.b0:slab * sh.b1] = np.asarray(pvp).reshape(-1)
        bs[sh.b0:sh.b1] = np.asarray(pbs).reshape(-1)
    return F2Tensor(f2, vp, bs, P, n_block)


# compute(local_records, local_block_id, local_n_block, f2_out, vpair_out) -> block_sizes.
# f2_out / vpair_out are flat float64 torch tensors of P*P*local_n_block values (CUDA on a
# GPU rank, CPU under gloo) that the compute fills; block_sizes comes back as int32 numpy.
ShardCompute = Callable[..., np.ndarray]


def extract_blocks_sharded(compute: ShardCompute, records, block_id, n_block: int, P: int, group=None,
                           device=None):
    """Sharded extraction across the ranks of `group` (torch.distributed; default group).

    Every rank computes its shard into its own buffers (rank 0 straight into its slice of the
    full output), then ranks 1.. send their slabs to rank 0, which receives them in place.
    All ranks take the same point-to-point steps, in rank order, whatever their shard; a rank
    with an empty shard sends nothing and rank 0 posts no receive for it. Returns
    (f2, vpair, block_sizes) as torch tensors on rank 0 (flat, P*P*n_block; block_sizes int32)
    and None elsewhere.

    A rank whose compute raises does not leave the others waiting in a receive: before the
    exchange every rank contributes an error flag to one all-reduce (MAX), and if any rank
    failed, all of them raise (the failing rank its own exception, chained), like the
    reference's fan-out rethrowing a worker's error (f2_blocks_multigpu_core.cpp:78-84).
    """
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = torch.device(device) if device is not None else torch.device("cpu")
    plan = plan_for(block_id, n_block, world)
    slab = P * P
    sh = plan[rank]

    if rank == 0:
        f2 = torch.zeros(slab * n_block, dtype=torch.float64, device=dev)
        vp = torch.zeros_like(f2)
        bs = torch.zeros(max(n_block, 0), dtype=torch.int32, device=dev)
        my_f2, my_vp = f2[slab * sh.b0:slab * sh.b1], vp[slab * sh.b0:slab * sh.b1]
    else:
        my_f2 = torch.zeros(slab * sh.n_block, dtype=torch.float64, device=dev)
        my_vp = torch.zeros_like(my_f2)
    my_bs = torch.zeros(max(sh.n_block, 0), dtype=torch.int32, device=dev)
    err = None
    if not sh.empty():
        try:
            b = compute(records[sh.s0:sh.s1], local_block_ids(block_id, sh), sh.n_block, my_f2, my_vp)
            my_bs.copy_(torch.from_numpy(np.ascontiguousarray(b, dtype=np.int32)).to(dev))
        except Exception as e:  # reported to every rank below, then re-raised here
            err = e
    flag = torch.tensor([0 if err is None else 1], dtype=torch.int32, device=dev)
    dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=group)
    if err is not None:
        raise RuntimeError(f"sharded extraction: rank {rank} failed on blocks [{sh.b0}, {sh.b1})") from err
    if int(flag.item()):
        raise RuntimeError("sharded extraction: another rank failed; no result was assembled")

    src_of = lambda r: dist.get_global_rank(group, r) if group is not None else r  # noqa: E731
    if rank == 0:
        if not sh.empty():
            bs[sh.b0:sh.b1] = my_bs
        for r in range(1, world):
            o = plan[r]
            if o.empty():
                continue
            dist.recv(f2[slab * o.b0:slab * o.b1], src=src_of(r), group=group)
            dist.recv(vp[slab * o.b0:slab * o.b1], src=src_of(r), group=group)
            dist.recv(bs[o.b0:o.b1], src=src_of(r), group=group)
        return f2, vp, bs
    if not sh.empty():
        dst = src_of(0)
        dist.send(my_f2, dst=dst, group=group)
        dist.send(my_vp, dst=dst, group=group)
        dist.send(my_bs, dst=dst, group=group)
    return None


def gpu_compute(ctx, records, n_ind: int, sel_rows, pop_offsets, precision=None, sample_ploidy=None,
                ploidy="auto") -> ShardCompute:
    """The per-rank compute on this rank's GPU through the C ABI (stp_f2_extract_blocks into
    device buffers). Unless sample_ploidy is given, ploidy is detected here once on the whole
    panel (stp_detect_ploidy over `records`' first min(1000, M) SNPs) and passed to every
    shard, as the reference decodes before it shards."""
    if sample_ploidy is None and str(ploidy) == "auto":
        sample_ploidy = ctx.detect_ploidy(records, n_ind, sel_rows)

    def run(local_records, local_block_id, local_n_block, f2_out, vp_out):
        _, _, bs = ctx.extract_blocks(local_records, n_ind, sel_rows, pop_offsets, local_block_id,
                                      local_n_block, precision=precision, sample_ploidy=sample_ploidy,
                                      ploidy=ploidy, out=(f2_out, vp_out))
        return bs

    return run
