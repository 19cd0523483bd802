"""Tile-class autotuner for the fixed-point contraction (the per-size-class choices the
reference makes in cuda_backend_f2_blocks.cu:55-74 and f2_batched_kernel.cu:31-74).

Measured here, per row class of an operand tile side (k: 8k+1 .. 8k+8 valid populations of
the tile's 128 rows): whether a pipeline stage copies the whole 36 KiB side (two bulk copies)
or only the side's valid 8-row groups of each of its nine planes (nine copies). For each
class it times the contraction of one request of 128 + rows populations (a full row tile and
a partial one: the full x partial and partial x partial tile pairs of every block) with the
class's bit set and cleared, on device-resident records, and keeps the faster. The table
goes to tile_classes.json beside this file; Context applies it (stp_set_tile_classes). The
other shape choices were measured once and are fixed (the M = 64 MMA costs what M = 128
does; the MMA width follows the column tile; split-K is never needed: every workload has
far more work items than SMs).

    python -m steppecu_b200.autotune [--snps 200000] [--reps 5]
"""
from __future__ import annotations

import argparse
import json
from pathlib import Path

TABLE = Path(__file__).resolve().parent / "tile_classes.json"
N_CLASSES = 16


def load_mask(default: int | None = None) -> int | None:
    """The committed partial-feed mask, or `default` when there is no table."""
    try:
        return int(json.loads(TABLE.read_text())["partial_feed_mask"])
    except (OSError, KeyError, ValueError):
        return default


def measure(snps: int = 200_000, reps: int = 5, device: int = 0) -> dict:
    import torch

    import steppecu_b200 as sb
    from steppecu_b200 import synth

    dev = f"cuda:{device}"
    panel = synth.generate("c2", seed=20261204, device=dev, n_snp=snps, n_pop=256)
    bpr = panel.bytes_per_record
    pitch = (bpr + 15) // 16 * 16
    rec = torch.zeros((panel.n_snp, pitch), dtype=torch.uint8, device=dev)
    rec[:, :bpr] = panel.records
    panel.records = None
    stream = torch.cuda.Stream(device=dev)
    rows_out = []
    with sb.Context(device) as ctx:
        for k in range(N_CLASSES):
            rows = 8 * k + 8
            P = 128 + rows
            sel, po = panel.selection(list(range(P)))
            plan = ctx.plan(rec, panel.n_ind, sel, po, panel.block_id, panel.n_block, precision="fixed_i8")
            f2 = torch.empty(P * P * panel.n_block, dtype=torch.float64, device=dev)
            vp = torch.empty_like(f2)
            ms = {}
            for partial in (False, True):
                mask = (1 << k) if partial else 0
                ctx.set_tile_classes(mask)
                for _ in range(2):
                    plan.run(rec, f2, vp, stream.cuda_stream)
                torch.cuda.synchronize()
                plan.set_timing(True)
                for _ in range(reps):
                    plan.run(rec, f2, vp, stream.cuda_stream)
                torch.cuda.synchronize()
                ms[partial] = plan.last_times()[1]
                plan.set_timing(False)
            plan.close()
            rows_out.append({"class": k, "rows": f"{8 * k + 1}-{rows}", "full_ms": ms[False], "partial_ms": ms[True],
                             "partial": bool(ms[True] < ms[False])})
        name = torch.cuda.get_device_name(device)
    mask = sum(1 << r["class"] for r in rows_out if r["partial"])
    return {"device": name, "snps": snps, "blocks": int(panel.n_block), "reps": reps,
            "measured": "contraction ms per pass (vpair + f2 kernels, CUDA events), request of 128 + rows populations",
            "classes": rows_out, "partial_feed_mask": mask}


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--snps", type=int, default=200_000)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=str(TABLE))
    args = ap.parse_args()
    table = measure(args.snps, args.reps)
    Path(args.out).write_text(json.dumps(table, indent=1) + "\n")
    print(json.dumps({"partial_feed_mask": table["partial_feed_mask"],
                      "classes": [(r["rows"], round(r["full_ms"], 4), round(r["partial_ms"], 4)) for r in table["classes"]]}))


if __name__ == "__main__":
    main()
