"""f2 block-tensor extraction benchmark (one JSON line on rank 0).

Metric: f2 SNP-pop-pairs/s = M * P*(P-1)/2 per extraction pass, per second. A step is one
pass of the hot path (ploidy -> decode -> per-block contraction -> FP64 f2/vpair) over
one synthetic panel already resident in HBM. Workload (default): 1,000 populations x 10
samples (10,000 total), 1,150,000 SNPs on 22 chromosomes, 5 cM blocks (~700), split-F16
tensor-core contraction (split-BF16 and the plain FP32 SIMT form are timed beside it). The panel (2.9 GB of genotypes, ~12 GB of operands) is far larger
than L2, so no flush is needed between steps.

`e2e` times the same extraction through the C ABI with host buffers: pinned genotypes in,
H2D copy, extraction, D2H of the FP64 f2 and vpair tensors, every step.

`--impl reference` times the reference's own CpuBackend (oracle/_ref, built from the
reference sources; the C restatement when that is absent) on the host cores, one
jackknife block per thread, on a bounded sample of the same workload. The same sample is
extracted on the GPU in every arithmetic and compared with it: `precision` reports the
max abs / rel f2 error against the reference at the workload's full population count.

Multi-GPU (torchrun): blocks are independent, so every rank extracts its own panel (a
different genome segment of the same shape): weak scaling, no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "f2 SNP·pop-pairs/s: split-BF16 TC vs plain FP32 on 1 B200, rel err ≤1e-6 vs FP64"
UNIT = "SNP·pop-pairs/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# The arithmetic each precision mode computes in (the bench line's dtype), and the operand
# bytes the decode writes per (population, SNP) in it.
DTYPES = {"split_bf16": "bf16x3", "split_f16": "f16x3", "split_f16_fine": "f16x3", "fixed_i8": "i8x4 (int32 exact)",
          "fp32": "f32"}
OPERAND_BYTES = {"split_bf16": 11, "split_f16": 11, "split_f16_fine": 11, "fixed_i8": 9, "fp32": 9}
# dram__bytes_read.sum + dram__bytes_write.sum per contraction (all its launches) at C3, from
# ncu captures summarised under profiles/ (split_f16: one pass on the full workload;
# fixed_i8: the 115k-SNP case scaled by its SNPs and blocks, 10x).
CONTRACTION_TRAFFIC = {("c3", "split_f16"): 13.58e9 + 12.24e9, ("c3", "fixed_i8"): 27.2e9 + 2.4e9}


def issued_tensor_work(P: int, block_id, n_block: int, con_ms: float, peak: float) -> dict:
    """Tensor work one split-arithmetic contraction launch issues, over its measured time.

    Every 32-SNP stage of a 128 x 128 tile pair (ti <= tj) issues 14 kind::f16 MMAs of
    128 x 128 x 16 (seven hi/lo products per 16 SNPs) and one kind::i8 MMA of 128 x 128 x 32
    (the exact vpair count). The algorithmic 6 * P^2 * M counts the full square of useful
    products once; the issued figure counts the split products, the triangle of tile pairs
    and the padding of P to tiles and of blocks to stages: it is what the tensor pipe runs.
    """
    import numpy as np

    k = np.bincount(np.asarray(block_id, np.int64), minlength=n_block)
    stages = int(((k + 31) // 32).sum())
    rt = (P + 127) // 128
    pairs = rt * (rt + 1) // 2
    f16 = pairs * stages * 14 * 2.0 * 128 * 128 * 16
    i8 = pairs * stages * 2.0 * 128 * 128 * 32
    sec = con_ms / 1000.0
    return {"f16_flops": f16, "i8_ops": i8, "f16_tflops": f16 / sec / 1e12, "f16_frac": f16 / sec / 1e12 / peak,
            "i8_tops": i8 / sec / 1e12}


def issued_fixed_work(P: int, block_id, n_block: int, con_ms: float, peak_bf16: float) -> dict:
    """Tensor work the fixed-point contraction issues, over its measured time (both kernels).

    Per 32-SNP stage of a 128 x 128 tile pair (ti <= tj): 18 kind::i8 MMAs of 128 x 128 x 32
    in the f2 kernel (ten digit products of X, four E(i) M(j), four M(i) E(j)) and one in the
    vpair kernel. The dense int8 tensor peak is twice the bf16 one on this part; the fraction
    is reported against twice the measured bf16 figure.
    """
    import numpy as np

    k = np.bincount(np.asarray(block_id, np.int64), minlength=n_block)
    stages = int(((k + 31) // 32).sum())
    rt = (P + 127) // 128
    pairs = rt * (rt + 1) // 2
    i8 = pairs * stages * 19 * 2.0 * 128 * 128 * 32
    sec = con_ms / 1000.0
    return {"i8_ops": i8, "i8_tops": i8 / sec / 1e12, "i8_frac": i8 / sec / 1e12 / (2.0 * peak_bf16),
            "peak_i8_tops": 2.0 * peak_bf16, "mmas_per_stage": 19}


def precision_all_blocks(f2_dev, vp_dev, rec_host, panel, sel, po, step: int = 10, threads: int | None = None,
                         rtol: float = 1e-6, atol: float = 1e-9) -> dict:
    """f2 error against the CPU oracle in every jackknife block of the full panel, on the pairs
    of every step-th population (step 10 at 1,000 populations: 100 of them, one in each 10,
    so their pairs fall in every 128 x 128 tile pair of the contraction; step 1: all pairs).
    f2 of a pair depends only on its two populations, so the oracle runs on that
    sub-selection: decode, then the per-block f2 on `threads` host threads."""
    import numpy as np
    import torch

    import oracle

    P, B = panel.n_pop, panel.n_block
    idx = np.arange(0, P, step)
    sub_sel = np.concatenate([sel[po[i]:po[i + 1]] for i in idx]).astype(np.int64)
    sub_po = np.concatenate([[0], np.cumsum([po[i + 1] - po[i] for i in idx])]).astype(np.int64)
    threads = threads or os.cpu_count() or 1
    t0 = time.perf_counter()
    pl = oracle.detect_ploidy_pa(rec_host, sub_sel)
    f2_ref, vp_ref, _ = oracle.f2_from_panel(rec_host, sub_sel, sub_po, panel.block_id, B, pl, threads=threads)
    cpu_s = time.perf_counter() - t0
    n = idx.size
    it = torch.as_tensor(idx, device=f2_dev.device)
    got = f2_dev.view(B, P, P).index_select(1, it).index_select(2, it).cpu().numpy().reshape(B, n, n)
    gvp = vp_dev.view(B, P, P).index_select(1, it).index_select(2, it).cpu().numpy().reshape(B, n, n)
    want = f2_ref.reshape(B, n, n)
    d = np.abs(got - want)
    a = np.abs(want)
    big = a >= 1e-12
    rel = np.where(big, d / np.where(big, a, 1.0), 0.0)
    per_abs = d.reshape(B, -1).max(axis=1)
    per_rel = rel.reshape(B, -1).max(axis=1)
    bad = d > atol + rtol * a
    return {
        "pairs": "every %d-th population: %d populations, %d pairs per block" % (step, n, n * (n - 1) // 2),
        "blocks": B, "oracle": "port (the C restatement: long-double pairwise sums, as the reference CpuBackend)",
        "oracle_seconds": cpu_s, "oracle_threads": threads,
        "max_abs": float(d.max()), "max_rel_f2_ge_1e-12": float(rel.max()),
        "max_comb_1e-9": float((d / (1e-9 + a)).max()),
        "max_rel_floor_1e-3": float((d / np.maximum(a, 1e-3)).max()),
        "tolerance": {"rtol": rtol, "atol": atol, "violations": int(bad.sum())},
        "vpair_bit_exact": bool(np.array_equal(gvp, vp_ref.reshape(B, n, n))),
        "per_block_max_abs": [float(x) for x in per_abs],
        "per_block_max_rel": [float(x) for x in per_rel],
    }


def run_fstats(ctx, f2, vp, block_id, P: int, B: int, n_stat: int = 100_000, reps: int = 3) -> dict:
    """f4 statistics with their block jackknife through stp_fstats on the device-resident f2
    tensor of the workload: the survivor pass over every slab's vpair, each quartet's
    per-block values from four f2 slabs, and the jackknife, for n_stat random quartets of
    distinct populations; the median of reps timed calls (host wall clock around the
    synchronous call, including the copy of est / var back). The CPU leg runs the reference
    CpuBackend's f-statistics (the port when the reference is absent) on one thread, on the
    sub-tensor of the first 40 populations (the per-statistic work does not depend on P)."""
    import numpy as np
    import torch

    import oracle
    from steppecu_b200 import _lib as L

    rng = np.random.default_rng(20261203)

    def quartets(n_pop, n):
        q = rng.integers(0, n_pop, size=(3 * n, 4))
        distinct = np.array([len(set(r)) == 4 for r in q.tolist()])
        return np.ascontiguousarray(q[distinct][:n], np.int32)

    bs = np.bincount(np.asarray(block_id, np.int64), minlength=B).astype(np.int32)
    q = quartets(P, n_stat)
    ctx.fstats(f2, vp, bs, P, B, L.FSTAT_F4, q.reshape(-1), q.shape[0])
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.fstats(f2, vp, bs, P, B, L.FSTAT_F4, q.reshape(-1), q.shape[0])
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)

    sub, n_cpu = min(40, P), 20_000
    f2s = f2.view(B, P, P)[:, :sub, :sub].contiguous().cpu().numpy().reshape(-1)
    vps = vp.view(B, P, P)[:, :sub, :sub].contiguous().cpu().numpy().reshape(-1)
    qc = quartets(sub, n_cpu)
    lib = "ref" if oracle.ref_available() else "port"
    t0 = time.perf_counter()
    oracle.fstats(f2s, vps, bs, sub, B, "f4", qc.reshape(-1), qc.shape[0], lib=lib)
    tc = time.perf_counter() - t0
    unit = "f4 statistics/s (with block jackknife)"
    return {"statistics": int(q.shape[0]), "blocks": B, "ms": 1000.0 * t, "value": q.shape[0] / t, "unit": unit,
            "cpu_baseline": {"value": qc.shape[0] / tc, "unit": unit, "cores": 1,
                             "kind": "reference" if lib == "ref" else "port",
                             "sample": f"{qc.shape[0]} quartets over the first {sub} populations, {B} blocks, one thread"}}


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling (every 200 ms) during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        try:
            rows = [ln.split(",") for ln in Path(self.f.name).read_text().splitlines() if ln.strip()]
        except OSError:
            rows = []
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, r[4:8]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def units(P: int, M: int) -> float:
    return float(M) * P * (P - 1) / 2.0


def host_d2h_bytes(P: int, B: int, wide: bool = False, tile: int = 128) -> int:
    """Bytes the host-output extraction downloads per call: the upper tile x tile tiles (row
    tile <= column tile, diagonal tiles whole) of every f2 slab in FP64, and of every vpair
    slab as packed 16-bit counts (32-bit when a block has 65,536 SNPs or more; packed tiles
    are whole tile x tile squares)."""
    t = -(-P // tile)
    upper = sum(min(tile, P - r0) * (P - r0) for r0 in range(0, P, tile))
    return 8 * B * upper + (4 if wide else 2) * B * (t * (t + 1) // 2) * tile * tile


def make_panel(workload: str, rank: int, device: str, n_snp: int | None = None):
    from steppecu_b200 import synth

    return synth.generate(workload, seed=20261203 + 1000 * rank, device=device, n_snp=n_snp)


def cpu_sample(workload: str, threads: int, seed_rank: int = 0, gen_device: str = "cpu", keep: bool = False):
    """Bounded CPU sample: `threads` blocks of the workload's panel model (one per thread),
    decoded and reduced by the CPU implementation. Returns (units, seconds, kind, desc) and,
    with keep=True, also (panel, block ids, f2, vpair) for the precision check."""
    import numpy as np

    import oracle
    from steppecu_b200 import synth

    wl = synth.WORKLOADS[workload]
    per_block = max(1, wl.n_snp // 700)
    n_snp = per_block * threads
    p = synth.generate(workload, seed=20261203 + 17 + seed_rank, device=gen_device, n_snp=n_snp)
    sel, po = p.selection()
    rec = p.records_numpy()
    bid = np.minimum(np.arange(n_snp) // per_block, threads - 1).astype(np.int32)
    kind = "reference" if oracle.ref_available() else "port"
    lib = "ref" if kind == "reference" else "port"
    t0 = time.perf_counter()
    if lib == "ref":
        # The reference end to end: its CpuBackend detects ploidy and decodes q / v / n from
        # the canonical individual-major tile (cpu_backend.cpp:73-95, 267-319), then reduces
        # the blocks (:217-264). Laying the records out as that tile is the reference's
        # reader's job (GenoReader); here the C restatement does it, inside the timing.
        tile, bpr_c = oracle.transpose_pa_to_canonical(rec, sel)
        q, v, nd = oracle.decode_af_canonical(tile, bpr_c, n_snp, po, detect=True, lib="ref")
    else:
        pl = oracle.detect_ploidy_pa(rec, sel)
        ac2, n = oracle.decode_counts_pa(rec, sel, po, pl)
        q, v, nd = oracle.counts_to_qvn(ac2, n)
    f2, vp, _ = oracle.compute_f2_blocks_sharded(q, v, nd, p.n_pop, bid, threads, threads=threads, lib=lib)
    dt = time.perf_counter() - t0
    legs = ("ploidy detection, decode and f2 by the reference CpuBackend (records laid out as its canonical "
            "tile by the C restatement)" if lib == "ref" else "decode and f2 by the C restatement")
    desc = (f"{threads} blocks x {per_block} SNPs of the {workload} panel model (P={p.n_pop}, "
            f"N={p.n_ind}); {legs}; f2 on {threads} threads, one block per thread")
    if keep:
        return units(p.n_pop, n_snp), dt, kind, desc, (p, bid, threads, f2, vp)
    return units(p.n_pop, n_snp), dt, kind, desc


def precision_report(ctx, sample, modes) -> dict:
    """GPU extraction of the CPU sample in each arithmetic against the CPU result."""
    import numpy as np

    p, bid, nb, f2_ref, vp_ref = sample
    sel, po = p.selection()
    rec = p.records_numpy()
    a = np.abs(f2_ref)
    big, sig = a >= 1e-12, a >= 1e-2
    out = {}
    for mode in modes:
        t = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, nb, precision=mode)
        d = np.abs(t.f2 - f2_ref)
        # Relative error is unbounded where a block's f2 estimate crosses zero, in every
        # arithmetic; max_rel_f2_ge_0.01 is the relative error over non-degenerate values.
        out[mode] = {"max_abs": float(d.max()), "max_rel": float((d[big] / a[big]).max()),
                     "max_rel_f2_ge_0.01": float((d[sig] / a[sig]).max()),
                     # the reference's combined check: |c - r| / (1e-9 + |r|)
                     "max_comb": float((d / (1e-9 + a)).max()),
                     "frac_f2_ge_0.01": float(sig.mean()),
                     "vpair_bit_exact": bool(np.array_equal(t.vpair, vp_ref)),
                     "vpair_mismatches": int(np.count_nonzero(t.vpair != vp_ref))}
        if mode == modes[0]:
            # Per jackknife block of the sample (slab b = the block's P x P values).
            slab = p.n_pop * p.n_pop
            db, ab, sb = d.reshape(nb, slab), a.reshape(nb, slab), sig.reshape(nb, slab)
            out[mode]["per_block"] = {
                "max_abs": [float(x) for x in db.max(axis=1)],
                "max_rel_f2_ge_0.01": [float((db[b][sb[b]] / ab[b][sb[b]]).max(initial=0.0)) for b in range(nb)],
            }
    return out


def run_reference(args, rank: int, world: int):
    threads = os.cpu_count() or 1
    if rank != 0:
        return
    for _ in range(args.warmup):
        cpu_sample(args.workload, threads)
    tot_u, tot_t = 0.0, 0.0
    kind, desc = "port", ""
    for _ in range(args.steps):
        u, t, kind, desc = cpu_sample(args.workload, threads)
        tot_u += u
        tot_t += t
    val = tot_u / tot_t
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "sample": desc},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": kind, "sample": desc},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_e2e(args, ctx, rec, panel, sel, po, bpr, n_out, barrier, dist, dev, P, M, B, world):
    """End to end through the C ABI with pinned host buffers: H2D of the genotypes,
    extraction, D2H of the FP64 f2 and vpair tensors, every step."""
    import numpy as np
    import torch

    rec_h = torch.empty((M, bpr), dtype=torch.uint8, pin_memory=True)
    rec_h.copy_(rec[:, :bpr])
    f2_h = torch.empty(n_out, dtype=torch.float64, pin_memory=True)
    vp_h = torch.empty(n_out, dtype=torch.float64, pin_memory=True)
    rec_np, f2_np, vp_np = rec_h.numpy(), f2_h.numpy(), vp_h.numpy()
    e2e_steps = args.e2e_steps or max(1, min(args.steps, 5))
    ctx.extract_blocks(rec_np, panel.n_ind, sel, po, panel.block_id, B, precision=args.precision,
                       out=(f2_np, vp_np))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.extract_blocks(rec_np, panel.n_ind, sel, po, panel.block_id, B, precision=args.precision,
                           out=(f2_np, vp_np))
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    # Host output through the tensor-core path: the upper tiles of every (exactly symmetric)
    # slab cross PCIe, f2 in FP64 and vpair as packed counts; the library fills the rest.
    segmented = args.precision != "fp32" and B >= 2 and P > 0
    wide = int(np.bincount(panel.block_id).max()) > 65535 if segmented else False
    d2h = host_d2h_bytes(P, B, wide) if segmented else 2 * n_out * 8
    e2e = {"value": units(P, M) * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(rec_h.numel()),
           "d2h_bytes_per_step": int(d2h), "output_bytes_per_step": int(2 * n_out * 8),
           "ms_per_step": 1000.0 * e2e_s, "steps": e2e_steps}

    return e2e


def run_config(workload: str, dev: str, modes, steps: int = 3, per_block: bool = False,
               precision_threads: int = 0) -> dict:
    """One of the other panel configs at full size on the device (records resident in HBM):
    each arithmetic as one persistent launch over all blocks, optionally also one launch per
    block, and optionally its precision against the CPU reference on a bounded block sample."""
    import torch

    import steppecu_b200 as sb
    from steppecu_b200 import synth

    panel = synth.generate(workload, seed=20261203 + 100 + int(workload[1]), device=dev)
    sel, po = panel.selection()
    P, M, B = panel.n_pop, panel.n_snp, panel.n_block
    bpr = panel.bytes_per_record
    pitch = (bpr + 15) // 16 * 16
    rec = torch.zeros((M, pitch), dtype=torch.uint8, device=dev)
    rec[:, :bpr] = panel.records
    panel.records = None
    f2 = torch.empty(P * P * B, dtype=torch.float64, device=dev)
    vp = torch.empty_like(f2)
    stream = torch.cuda.Stream(device=dev)
    ctx = sb.Context(int(dev.split(":")[1]) if ":" in dev else 0)
    counts = torch.bincount(torch.as_tensor(panel.block_id), minlength=B)
    out = {"populations": P, "samples": panel.n_ind, "snps": M, "blocks": B,
           "block_snps": {"min": int(counts.min()), "median": int(counts.median()), "max": int(counts.max())}}

    def timed(plan, n):
        plan.run(rec, f2, vp, stream.cuda_stream)
        torch.cuda.synchronize()
        plan.set_timing(True)
        l0 = ctx.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            plan.run(rec, f2, vp, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        dec, con = plan.last_times()
        plan.set_timing(False)
        return e0.elapsed_time(e1) / n, dec, con, (ctx.launches - l0) / n

    for mode in modes:
        plan = ctx.plan(rec, panel.n_ind, sel, po, panel.block_id, B, precision=mode)
        ms, dec, con, nl = timed(plan, steps)
        r = {"value": units(P, M) / (ms / 1e3), "ms_per_step": ms, "decode_ms": dec, "contract_ms": con,
             "launches_per_step": nl}
        if per_block and mode != "fp32":
            plan.set_per_block_launch(True)
            ms_b, _, con_b, nl_b = timed(plan, steps)
            plan.set_per_block_launch(False)
            r["per_block_launches"] = {"ms_per_step": ms_b, "contract_ms": con_b, "launches_per_step": nl_b,
                                       "persistent_speedup": ms_b / ms}
        plan.close()
        out[mode] = r
    if precision_threads:
        u, t, kind, desc, sample = cpu_sample(workload, precision_threads, gen_device=dev, keep=True)
        out["cpu_baseline"] = {"value": u / t, "unit": UNIT, "cores": precision_threads, "kind": kind, "sample": desc}
        out["precision"] = precision_report(ctx, sample, modes)
    ctx.close()
    return out


def run_batched(dev: str, steps: int = 3, n_req: int = 64, serial_baselines: bool = True, warmup: int = 3,
                precision: str = "split_f16") -> dict:
    """Many requests over one shared panel (8,000 samples x 1.15M SNPs, 64 requests of
    4-300 populations, each with its own 5 cM block map): one grouped stp_f2_extract_batch
    call against the same requests extracted one after another (plain FP32 SIMT and
    split-F16). Records and outputs stay in HBM; each call is synchronous and timed on the
    host around it (its planning is part of the cost); per-request completion times of the
    grouped call come from device stamps."""
    import numpy as np
    import torch

    import steppecu_b200 as sb
    from steppecu_b200 import synth

    panel = synth.generate("c5", seed=20261203 + 5, device=dev)
    reqs = synth.batch_requests(panel, n_req=n_req)
    M = panel.n_snp
    bpr = panel.bytes_per_record
    pitch = (bpr + 15) // 16 * 16
    rec = torch.zeros((M, pitch), dtype=torch.uint8, device=dev)
    rec[:, :bpr] = panel.records
    panel.records = None
    Ps = [len(q["pop_offsets"]) - 1 for q in reqs]
    total_units = sum(units(P, M) for P in Ps)
    outs = []
    for q, P in zip(reqs, Ps):
        n = P * P * q["n_block"]
        outs.append((torch.empty(n, dtype=torch.float64, device=dev), torch.empty(n, dtype=torch.float64, device=dev)))
    ordinal = int(dev.split(":")[1]) if ":" in dev else 0

    def serial(ctx, precision: str):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        comp = []
        for q, (f2, vp) in zip(reqs, outs):
            ctx.extract_blocks(rec, panel.n_ind, q["sel_rows"], q["pop_offsets"], q["block_id"], q["n_block"],
                               precision=precision, out=(f2, vp))
            comp.append((time.perf_counter() - t0) * 1e3)
        return comp

    def serial_median(ctx, precision: str, passes: int = 3):
        # The pass with the median total (single passes vary with the device allocations of
        # the per-request plans).
        runs = sorted((serial(ctx, precision) for _ in range(passes)), key=lambda c: c[-1])
        return runs[len(runs) // 2]

    # Serial baselines first, each on a fresh context (no workspace of another form held).
    ser_f32 = ser_f16 = ref = None
    if serial_baselines:
        ctx = sb.Context(ordinal)
        serial(ctx, "fp32")  # warm-up
        ser_f32 = serial_median(ctx, "fp32")
        ctx.close()
        ctx = sb.Context(ordinal)
        serial(ctx, precision)  # warm-up
        ser_f16 = serial_median(ctx, precision)
        ref = [(f2.clone(), vp.clone()) for f2, vp in outs]
        ctx.close()

    ctx = sb.Context(ordinal)

    def grouped():
        torch.cuda.synchronize()
        t = time.perf_counter()
        ctx.extract_batch(rec, panel.n_ind, reqs, precision=precision, out=outs)
        return time.perf_counter() - t

    for _ in range(max(1, warmup)):  # warm-up (the first call allocates the batch workspace)
        grouped()
    l0 = ctx.launches
    wall = [grouped() for _ in range(steps)]
    launches = (ctx.launches - l0) / steps
    done = ctx.last_batch_times(len(reqs))
    same = None if ref is None else all(torch.equal(a, c) and torch.equal(b, d) for (a, b), (c, d) in zip(ref, outs))
    ctx.close()
    med = float(np.median(wall))

    def pct(x, p):
        return float(np.percentile(np.asarray(x), p))

    return {
        "workload": "c5: 64 requests over one panel of 8,000 samples (400 pops x 20) x 1.15M SNPs",
        "requests": len(reqs), "populations_per_request": {"min": min(Ps), "max": max(Ps), "sum_sq": int(sum(P * P for P in Ps))},
        "units": total_units,
        "grouped": {"value": total_units / med, "unit": UNIT, "ms_per_call": med * 1e3, "calls": steps,
                    "device_span_ms": float(np.nanmax(done)),
                    "device_value": total_units / (float(np.nanmax(done)) / 1e3),
                    "completion_ms_p50": pct(done, 50), "completion_ms_p99": pct(done, 99), "gpu_launches": launches,
                    "precision": precision, "equals_serial": same},
        "serial_same_precision": None if ser_f16 is None else {
            "value": total_units / (ser_f16[-1] / 1e3), "ms_total": ser_f16[-1],
            "completion_ms_p50": pct(ser_f16, 50), "completion_ms_p99": pct(ser_f16, 99)},
        "serial_fp32": None if ser_f32 is None else {
            "value": total_units / (ser_f32[-1] / 1e3), "ms_total": ser_f32[-1],
            "completion_ms_p50": pct(ser_f32, 50), "completion_ms_p99": pct(ser_f32, 99)},
        "timing": "host wall clock around each synchronous call (serial: the median of three passes); completion of "
                  "grouped requests from device stamps",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c5: only the many-requests measurement (grouped batch vs serial)")
    ap.add_argument("--precision", default="fixed_i8")
    ap.add_argument("--also", default="split_f16,split_bf16,split_f16_fine",
                    help="other tensor-core arithmetics timed beside the headline (comma-separated, or none)")
    ap.add_argument("--compare-simt", action="store_true", default=True)
    ap.add_argument("--no-compare-simt", dest="compare_simt", action="store_false")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-threads", type=int, default=None)
    ap.add_argument("--snps", type=int, default=None, help="override the workload's SNP count (smaller cases)")
    ap.add_argument("--quick", action="store_true", help="headline timing only: no other arithmetics, e2e or CPU leg")
    ap.add_argument("--no-batched", dest="batched", action="store_false",
                    help="skip the many-requests (grouped batch) measurement")
    ap.add_argument("--no-other-configs", dest="other_configs", action="store_false",
                    help="skip the 100-population and uneven-block config measurements")
    ap.add_argument("--block-snps", type=int, default=None,
                    help="uniform jackknife blocks of this many SNPs instead of the 5 cM walk (profiling cases: "
                         "--snps 115000 --block-snps 1611 keeps the headline block size at a tenth of the SNPs)")
    ap.add_argument("--precision-step", type=int, default=10,
                    help="per-block f2 error of the headline pass against the CPU oracle on the pairs of every "
                         "n-th population, all blocks (1: all pairs, several minutes of host time at 1,000 "
                         "populations; 0: skip)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    args.warmup = max(3, args.warmup)

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch

    import steppecu_b200 as sb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    dev = f"cuda:{local}"
    if args.workload == "c5":
        b = run_batched(dev, steps=args.steps, serial_baselines=not args.quick, warmup=args.warmup,
                        precision=args.precision)
        if rank == 0:
            print(json.dumps({
                "metric": METRIC, "value": b["grouped"]["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": b["grouped"]["ms_per_call"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": DTYPES.get(args.precision, "f32"), "data": "synthetic",
                "config": {"workload": "c5", "requests": b["requests"], "samples": 8000, "snps": 1150000,
                           "precision": args.precision, "parallelism": "1 GPU"},
                "gpu_launches": b["grouped"]["gpu_launches"], "batched_requests": b}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    panel = make_panel(args.workload, rank, dev, n_snp=args.snps)
    if args.block_snps:
        import numpy as np

        panel.block_id = (np.arange(panel.n_snp) // args.block_snps).astype(np.int32)
        panel.n_block = int(panel.block_id[-1]) + 1 if panel.n_snp else 0
    sel, po = panel.selection()
    P, M, B = panel.n_pop, panel.n_snp, panel.n_block
    ctx = sb.Context(local)
    # Device-resident records at a 16-byte pitch (128-bit loads); bytes_per_record stays bpr.
    bpr = panel.bytes_per_record
    pitch = (bpr + 15) // 16 * 16
    rec = torch.zeros((M, pitch), dtype=torch.uint8, device=dev)
    rec[:, :bpr] = panel.records
    panel.records = None
    n_out = P * P * B
    f2 = torch.empty(n_out, dtype=torch.float64, device=dev)
    vp = torch.empty_like(f2)
    # A dedicated stream: the library and the CUDA events must see the same stream handle
    # (torch's legacy default stream has handle 0, which the C ABI reads as "context stream").
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    plan = ctx.plan(rec, panel.n_ind, sel, po, panel.block_id, B, precision=args.precision)

    def timed(pl, steps, warm):
        for _ in range(warm):
            pl.run(rec, f2, vp, stream.cuda_stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        pl.set_timing(True)
        l0 = ctx.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            pl.run(rec, f2, vp, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.launches - l0
        ms = e0.elapsed_time(e1) / steps
        dec, con = pl.last_times()
        pl.set_timing(False)
        barrier()
        return ms, dec, con, launches

    def timed_graph(pl, steps, warm):
        # The pass replayed from one CUDA graph (ploidy, transpose, decode, contraction).
        for _ in range(warm):
            pl.run_graph(rec, f2, vp, stream.cuda_stream)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        l0 = ctx.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            pl.run_graph(rec, f2, vp, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.launches - l0
        barrier()
        return e0.elapsed_time(e1) / steps, launches

    with Clocks(local) as clk:
        ms, launches = timed_graph(plan, args.steps, args.warmup)
        # Per-kernel split (decode vs contraction) from event-bracketed plain runs.
        _, dec_ms, con_ms, _ = timed(plan, args.steps, args.warmup)
    clocks = clk.summary()
    # The headline pass's f2 against the CPU oracle in every block (before other plans reuse
    # the output buffers).
    prec_all = None
    if rank == 0 and world == 1 and not args.quick and args.precision_step > 0:
        rec_host = rec[:, :bpr].cpu().numpy()
        prec_all = precision_all_blocks(f2, vp, rec_host, panel, sel, po, step=args.precision_step,
                                        threads=args.cpu_threads)
        prec_all["precision"] = args.precision
        del rec_host
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = units(P, M) * world / (ms / 1000.0)

    # The other arithmetics on the same panel: the plain FP32 SIMT form (the comparison the
    # metric names) and the other tensor-core split.
    others = {}
    extra = []
    if args.compare_simt and args.precision != "fp32" and not args.quick:
        extra.append("fp32")
    if args.also and not args.quick:
        extra += [m for m in args.also.split(",") if m and m not in (args.precision, "none")]
    for prec in extra:
        plan_s = ctx.plan(rec, panel.n_ind, sel, po, panel.block_id, B, precision=prec)
        s_steps = max(1, min(args.steps, 3))
        ms_s, dec_s, con_s, _ = timed(plan_s, s_steps, 1)
        others[prec] = {"value": units(P, M) * world / (ms_s / 1000.0), "ms_per_step": ms_s,
                        "contract_ms": con_s, "decode_ms": dec_s}
        plan_s.close()

    # The grouped schedule against one contraction launch per jackknife block.
    per_block = None
    if args.precision != "fp32" and not args.quick:
        plan.set_per_block_launch(True)
        ms_b, dec_b, con_b, l_b = timed(plan, max(1, min(args.steps, 3)), 1)
        plan.set_per_block_launch(False)
        per_block = {"ms_per_step": ms_b, "contract_ms": con_b, "launches_per_step": l_b / max(1, min(args.steps, 3)),
                     "value": units(P, M) * world / (ms_b / 1000.0)}

    fst = None
    if not args.quick and rank == 0 and world == 1 and P >= 4:
        fst = run_fstats(ctx, f2, vp, panel.block_id, P, B)

    e2e = None
    if not args.quick:
        e2e = run_e2e(args, ctx, rec, panel, sel, po, bpr, n_out, barrier, dist, dev, P, M, B, world)

    # Roofline of the dominant kernel (the contraction): algorithmic flops per launch =
    # 3 contractions x 2 * P^2 * M (SNP-padded work excluded) over the measured launch time.
    peaks, peak_kind = load_peaks()
    flops = 6.0 * P * P * M
    achieved = flops / (con_ms / 1000.0) / 1e12
    peak = float(peaks.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"]))
    # DRAM bytes (read + write) of one contraction launch on this workload, from one ncu
    # capture of it (summarised under profiles/).
    traffic = CONTRACTION_TRAFFIC.get((args.workload, args.precision)) if args.snps is None else None
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "kernel_ms": con_ms, "decode_ms": dec_ms,
                "decode_hbm_gbs": (M * bpr + OPERAND_BYTES.get(args.precision, 11) * P * M) / (dec_ms / 1000.0) / 1e9}
    if args.precision == "fixed_i8":
        roofline["issued"] = issued_fixed_work(P, panel.block_id, B, con_ms, peak)
    elif args.precision != "fp32":
        roofline["issued"] = issued_tensor_work(P, panel.block_id, B, con_ms, peak)

    cpu = None
    precision = None
    if rank == 0 and world == 1 and not args.quick:
        threads = args.cpu_threads or (os.cpu_count() or 1)
        u, t, kind, desc, sample = cpu_sample(args.workload, threads, gen_device=dev, keep=True)
        cpu = {"value": u / t, "unit": UNIT, "cores": threads, "kind": kind, "sample": desc}
        if threads > 1:  # the same implementation on one core: one block of the same model
            u1, t1, _, desc1 = cpu_sample(args.workload, 1, seed_rank=1, gen_device=dev)
            cpu["single_core"] = {"value": u1 / t1, "unit": UNIT, "cores": 1, "sample": desc1}
        modes = [args.precision] + [m for m in ("fixed_i8", "split_f16", "split_f16_fine", "split_bf16", "fp32")
                                    if m != args.precision]
        precision = {"against": f"{kind} CPU f2 on the cpu_baseline sample", **precision_report(ctx, sample, modes)}

    other_configs = None
    if world == 1 and not args.quick and args.other_configs:
        # The full-panel plain GPU form (100 pops x 20) and the uneven-blocks config (1,000
        # lognormal pops, lognormal blocks): full size, records in HBM.
        threads = args.cpu_threads or (os.cpu_count() or 1)
        other_configs = {
            "c2": run_config("c2", dev, ["fp32", "fixed_i8", "split_f16"], precision_threads=threads),
            "c4": run_config("c4", dev, ["fixed_i8", "split_f16", "split_bf16"], per_block=True),
        }

    batched = None
    if world == 1 and not args.quick and args.batched:
        plan.close()
        ctx.close()
        del rec, f2, vp, plan, ctx
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        batched = run_batched(dev, warmup=args.warmup, precision=args.precision)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPES.get(args.precision, "f32"),
            "data": "synthetic",
            "config": {"workload": args.workload, "populations": P, "samples": panel.n_ind, "snps": M,
                       "blocks": B, "block_snps": args.block_snps or "5 cM walk", "precision": args.precision, "l2": "inputs larger than L2 (no flush)",
                       "cuda_graph": True,
                       "parallelism": f"block-sharded x{world}" if world > 1 else "1 GPU"},
            "gpu_launches": int(launches), "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
            # The same throughput counted over ordered population pairs with the diagonal
            # (M * P^2 per pass), the other convention for this metric.
            "value_ordered_pairs": {"value": value * 2.0 * P / (P - 1) if P > 1 else None,
                                    "unit": "SNP·ordered-pop-pairs/s (P^2 per SNP)"},
            "precision": precision,
            "precision_all_blocks": prec_all,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "other_arithmetics": others,
            "per_block_launches": per_block, "fstats": fst,
            "batched_requests": batched,
            "other_configs": other_configs,
        }
        print(json.dumps(line), flush=True)
    if batched is None:
        plan.close()
        ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
