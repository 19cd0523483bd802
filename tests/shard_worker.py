"""One gloo rank of the sharded-extraction tests (started with the `spawn` method).

Each rank draws the same seeded panel, extracts its block shard with the oracle standing in
for the GPU compute, and takes part in steppecu_b200.shard.extract_blocks_sharded's
exchange. Rank 0 writes the assembled tensor (or each rank its error) to out_dir.
"""
from __future__ import annotations

import datetime
import os
import sys
import traceback
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def panel_case(case: str):
    """(records, sel, pop_offsets, block_id, n_block, P, ploidy) for a named case."""
    import numpy as np

    import oracle
    from steppecu_b200 import synth

    p = synth.generate("c4", seed=11, n_snp=5000, n_pop=9)
    rec = p.records_numpy()
    sel, po = p.selection()
    bid, nb = np.asarray(p.block_id, np.int32), int(p.n_block)
    if case == "two_blocks":  # fewer blocks than ranks: trailing empty shards
        bid = (np.arange(rec.shape[0]) >= 3100).astype(np.int32)
        nb = 2
    pl = oracle.detect_ploidy_pa(rec, sel)
    return rec, sel, po, bid, nb, len(po) - 1, pl


def run(rank: int, world: int, port: int, case: str, out_dir: str, fail_rank: int = -1) -> None:
    import numpy as np
    import torch
    import torch.distributed as dist

    import oracle
    from steppecu_b200 import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    out = Path(out_dir)
    try:
        rec, sel, po, bid, nb, P, pl = panel_case(case)
        seen = []

        def compute(lrec, lbid, lnb, f2_out, vp_out):
            if rank == fail_rank:
                raise ValueError("injected failure")
            seen.append((int(lrec.shape[0]), int(lnb), int(lbid.min()), int(lbid.max())))
            f2, vp, bs = oracle.f2_from_panel(lrec, sel, po, lbid, lnb, pl)
            f2_out.copy_(torch.from_numpy(f2))
            vp_out.copy_(torch.from_numpy(vp))
            return bs

        try:
            res = shard.extract_blocks_sharded(compute, rec, bid, nb, P)
        except RuntimeError as e:
            (out / f"error{rank}.txt").write_text(str(e))
            return
        np.save(out / f"seen{rank}.npy", np.asarray(seen, np.int64).reshape(-1, 4))
        if rank == 0:
            f2, vp, bs = res
            np.savez(out / "got.npz", f2=f2.numpy(), vpair=vp.numpy(), block_sizes=bs.numpy())
        else:
            assert res is None
    except Exception:
        (out / f"crash{rank}.txt").write_text(traceback.format_exc())
        raise
    finally:
        dist.destroy_process_group()
