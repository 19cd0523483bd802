"""extract-f2's SNP filters on the device (stp_snp_keep_mask) and the fused compaction
(stp_f2_request.kept_rows) against the CPU oracle.

The keep mask and the pooled per-SNP summary are compared bit for bit with the oracle's
or_keep_mask (itself pinned to the reference's keep_decision_pooled in
test_filters_oracle.py) over the oracle's own decode; an extraction over kept rows read in
place must equal the extraction over a compacted copy of the records, bit for bit, and the
oracle within the arithmetic's tolerance.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from steppecu_b200 import F2Tensor, extract_f2, synth
from steppecu_b200.blocks import assign_blocks
from steppecu_b200.synth import write_eigenstrat

pytestmark = pytest.mark.gpu

ACGT = np.frombuffer(b"ACGT", np.uint8)


def _snp_columns(M: int, seed: int):
    rng = np.random.default_rng(seed)
    ref = ACGT[rng.integers(0, 4, M)]
    alt = ACGT[rng.integers(0, 4, M)]                 # some equal to ref: multiallelic
    alt[rng.random(M) < 0.02] = ord("N")
    ref[rng.random(M) < 0.01] = ord("c")              # lower case counts as the base
    chrom = rng.integers(1, 25, M).astype(np.int32)  # 23, 24: not autosomes
    return ref, alt, chrom


@pytest.fixture(scope="module")
def panel():
    p = synth.generate("c2", seed=31, n_snp=30_000, n_pop=41)
    sel, po = p.selection()
    rec = p.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = oracle.decode_counts_pa(rec, sel, po, pl)
    q, _, nd = oracle.counts_to_qvn(ac2, n)
    return p, sel, po, rec, pl, q, nd


FILTERS = [
    dict(),
    dict(maf_min=0.05, maxmiss=0.2, strand_mode="drop"),
    dict(maf_min=0.01, maxmiss=0.0, autosomes_only=True, drop_monomorphic=True, strand_mode="keep"),
    dict(transversions_only=True, strand_mode="flip", maxmiss=0.5),
]


@pytest.mark.parametrize("filt", FILTERS)
def test_keep_mask_equals_oracle(ctx, panel, filt):
    p, sel, po, rec, pl, q, nd = panel
    ref, alt, chrom = _snp_columns(p.n_snp, 7)
    keep, summ = ctx.snp_keep_mask(rec, p.n_ind, sel, po, ref, alt, chrom, summary=True, **filt)
    strand = {"drop": 0, "keep": 1, "flip": 2}[filt.get("strand_mode", "drop")]
    kw = {k: v for k, v in filt.items() if k != "strand_mode"}
    want, wsum = oracle.keep_mask(q, nd, p.n_pop, ref, alt, chrom, strand_mode=strand,
                                  total_indiv=float(po[-1]), **kw)
    assert np.array_equal(keep, want.astype(bool)), int((keep != want.astype(bool)).sum())
    assert np.array_equal(summ, wsum)
    assert 0 < keep.sum() < p.n_snp or not filt


@pytest.mark.parametrize("mode", ["split_f16", "fixed_i8"])
def test_kept_rows_equal_compacted_records(ctx, panel, mode):
    import torch

    p, sel, po, rec, pl, _, _ = panel
    rng = np.random.default_rng(3)
    idx = np.flatnonzero(rng.random(p.n_snp) < 0.7)
    idx = idx[idx >= 5]                                # the first records are read for ploidy only
    bid, nb = assign_blocks(p.chrom[idx], p.genpos[idx], 0.05, p.physpos[idx])
    compact = np.ascontiguousarray(rec[idx])
    want = ctx.extract_blocks(compact, p.n_ind, sel, po, bid, nb, precision=mode, sample_ploidy=pl)
    # Host records (segmented upload of the kept row ranges), auto ploidy on the raw records.
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, nb, precision=mode, kept_rows=idx)
    assert np.array_equal(got.f2, want.f2) and np.array_equal(got.vpair, want.vpair)
    assert np.array_equal(got.block_sizes, want.block_sizes)
    # Device records through a plan.
    d_rec = torch.as_tensor(rec).cuda()
    plan = ctx.plan(d_rec, p.n_ind, sel, po, bid, nb, precision=mode, kept_rows=idx)
    n = p.n_pop * p.n_pop * nb
    f2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    vp = torch.zeros(n, dtype=torch.float64, device="cuda")
    plan.run(d_rec, f2, vp)
    torch.cuda.synchronize()
    assert np.array_equal(f2.cpu().numpy(), want.f2) and np.array_equal(vp.cpu().numpy(), want.vpair)
    plan.close()
    # And the oracle on the compacted records, with the raw records' ploidy.
    of2, ovp, obs = oracle.f2_from_panel(compact, sel, po, bid, nb, pl, threads=8)
    assert np.array_equal(got.vpair, ovp)
    tol = (1e-6, 1e-9) if mode == "fixed_i8" else (5e-6, 2e-7)
    assert np.all(np.abs(got.f2 - of2) <= tol[1] + tol[0] * np.abs(of2))


def test_kept_rows_are_validated(ctx, panel):
    from steppecu_b200 import StpError

    p, sel, po, rec, _, _, _ = panel
    bid = np.zeros(3, np.int32)
    for bad in ([5, 4, 9], [0, 1, p.n_snp]):
        with pytest.raises(StpError, match="kept_rows"):
            ctx.extract_blocks(rec, p.n_ind, sel, po, bid, 1, precision="fixed_i8", kept_rows=np.array(bad))


def test_extract_f2_filtered_files_vs_oracle(tmp_path):
    """The whole front end from .geno/.snp/.ind with AT2-style filters: the device keep mask,
    the block walk over the kept SNPs, the extraction over kept rows in place."""
    p = synth.generate("c1", seed=77, n_snp=12_000, n_pop=8)
    write_eigenstrat(p, tmp_path / "panel")
    from steppecu_b200.eigenstrat import read_snp

    snp = read_snp(tmp_path / "panel.snp")
    pops = sorted(p.pop_labels)[:6]
    filt = dict(maf=0.05, maxmiss=0.0, autosomes_only=True, drop_monomorphic=True, strand_mode="drop")
    h = extract_f2(tmp_path / "panel", pops=pops, precision="fixed_i8", **filt)
    # Oracle: the same selection, mask, blocks and f2.
    labels = sorted(pops)
    order = [p.pop_labels.index(x) for x in labels]
    sel, po = p.selection(order)
    rec = p.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = oracle.decode_counts_pa(rec, sel, po, pl)
    q, _, nd = oracle.counts_to_qvn(ac2, n)
    keep, _ = oracle.keep_mask(q, nd, len(labels), snp.ref, snp.alt, snp.chrom, maf_min=0.05, maxmiss=0.0,
                               autosomes_only=True, drop_monomorphic=True, strand_mode=0,
                               total_indiv=float(po[-1]))
    idx = np.flatnonzero(keep)
    bid, nb = oracle.assign_blocks(snp.chrom[idx], snp.genpos[idx], 0.05, snp.physpos[idx])
    f2, vp, bs = oracle.f2_from_panel(np.ascontiguousarray(rec[idx]), sel, po, bid, nb, pl, threads=8)
    want = F2Tensor(f2, vp, bs, len(labels), nb)
    got = h.tensor
    assert got.n_block == nb and np.array_equal(got.block_sizes, bs)
    assert np.array_equal(got.vpair, vp)
    assert np.all(np.abs(got.f2 - f2) <= 1e-9 + 1e-6 * np.abs(f2))
    assert want.P == got.P
