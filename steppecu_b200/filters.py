"""SNP keep-mask for extract-f2 (the AT2 default filters of the reference's extract path).

Rules follow src/io/filter/filter_decision.hpp and keep_decision_pooled
(src/io/filter/snp_summary_reduce.hpp:38-81): multiallelic and (with strand_mode "drop")
strand-ambiguous SNPs are dropped, then pooled minor-allele frequency >= maf, optional
monomorphic drop, transversions-only, autosomes 1..22. The sample-axis missingness test
is disabled on this path and ``maxmiss`` is applied on the population axis instead: a SNP
is dropped when the fraction of selected populations with no called allele exceeds
maxmiss (src/app/extract_f2_core.cpp:246-263). Counts come from the GPU decode.
"""
from __future__ import annotations

import numpy as np

AUTOSOME_MIN, AUTOSOME_MAX = 1, 22
_ACGT = {ord("A"): "A", ord("C"): "C", ord("G"): "G", ord("T"): "T"}
_COMP = {"A": "T", "T": "A", "C": "G", "G": "C"}


def _norm(a: np.ndarray) -> np.ndarray:
    a = a.astype(np.uint8).copy()
    lower = (a >= ord("a")) & (a <= ord("z"))
    a[lower] -= 0x20
    ok = np.isin(a, [ord("A"), ord("C"), ord("G"), ord("T")])
    a[~ok] = 0
    return a


def metadata_keep(ref: np.ndarray, alt: np.ndarray, chrom: np.ndarray, *, autosomes_only: bool,
                  transversions_only: bool, strand_mode: str) -> np.ndarray:
    r, a = _norm(ref), _norm(alt)
    multi = (r == 0) | (a == 0) | (r == a)
    comp = np.zeros(256, np.uint8)
    for x, y in _COMP.items():
        comp[ord(x)] = ord(y)
    ambiguous = (~multi) & (r == comp[a])
    purine = np.zeros(256, bool)
    purine[[ord("A"), ord("G")]] = True
    transition = (~multi) & (purine[r] == purine[a])
    transversion = (~multi) & ~transition
    keep = ~multi
    if strand_mode == "drop":
        keep &= ~ambiguous
    if transversions_only:
        keep &= transversion
    if autosomes_only:
        keep &= (chrom >= AUTOSOME_MIN) & (chrom <= AUTOSOME_MAX)
    return keep


def snp_keep_mask(ctx, records, header, snp, sel_rows, pop_offsets, *, ploidy="auto", maf=0.0, maxmiss=0.0,
                  autosomes_only=True, drop_monomorphic=False, transversions_only=False, strand_mode="drop",
                  chunk: int = 1 << 16) -> np.ndarray:
    M = header.n_snp
    keep = metadata_keep(snp.ref[:M], snp.alt[:M], snp.chrom[:M], autosomes_only=autosomes_only,
                         transversions_only=transversions_only, strand_mode=strand_mode)
    need_counts = maf > 0.0 or drop_monomorphic or maxmiss < 1.0
    if not need_counts:
        return keep
    sample_ploidy = ctx.detect_ploidy(records, header.n_ind, sel_rows) if ploidy == "auto" else None
    P = len(pop_offsets) - 1
    for s0 in range(0, M, chunk):
        s1 = min(M, s0 + chunk)
        ac2, n = ctx.decode_counts(np.ascontiguousarray(records[s0:s1]), header.n_ind, sel_rows, pop_offsets,
                                   sample_ploidy=sample_ploidy, ploidy=ploidy)
        nd = n.astype(np.float64)
        q = np.where(n > 0, (ac2.astype(np.float64) * 0.5) / np.where(n > 0, nd, 1.0), 0.0)
        # Pooled reference frequency, summed in population order (derive_pooled_summary_one).
        ref_count = np.zeros(s1 - s0)
        allele_count = np.zeros(s1 - s0)
        for p in range(P):
            ref_count = ref_count + q[p] * nd[p]
            allele_count = allele_count + nd[p]
        pooled = np.where(allele_count > 0, ref_count / np.where(allele_count > 0, allele_count, 1.0), 0.0)
        minor = np.minimum(pooled, 1.0 - pooled)
        k = keep[s0:s1]
        k &= minor >= maf
        if drop_monomorphic:
            k &= minor != 0.0
        if maxmiss < 1.0:
            frac_missing_pops = (n <= 0).sum(axis=0) / float(P)
            k &= ~(frac_missing_pops > maxmiss)
        keep[s0:s1] = k
    return keep
