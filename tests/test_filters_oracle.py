"""extract-f2's SNP keep mask: the C restatement (oracle/f2_oracle.c or_keep_mask) against
the reference's own keep rule (io::filter::derive_pooled_summary_one + keep_decision_pooled,
src/io/filter/snp_summary_reduce.hpp:38-79, and the population-coverage bound of
extract_f2_core.cpp:245-259), compiled from the reference sources by oracle/Makefile. Masks
and pooled summaries must agree bit for bit, over every filter option."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import oracle

ALLELES = list("ACGTacgt") + ["N", "0", "-", "R"]


def _random_case(seed, P=13, M=4000):
    rng = np.random.default_rng(seed)
    n = rng.integers(0, 21, size=(M, P)).astype(np.int32)
    n[rng.random((M, P)) < 0.15] = 0                     # missing populations
    ac2 = np.minimum(rng.integers(0, 41, size=(M, P)), 2 * n).astype(np.int32)
    mono = rng.random(M) < 0.1                           # some SNPs monomorphic
    ac2[mono] = 0
    q, v, nd = oracle.counts_to_qvn(ac2.reshape(-1), n.reshape(-1))
    ref = rng.choice(ALLELES, size=M)
    alt = rng.choice(ALLELES, size=M)
    chrom = rng.integers(0, 26, size=M).astype(np.int32)
    return q, nd, P, ref, alt, chrom, int(rng.integers(P * 5, P * 15))


@pytest.mark.skipif(not oracle.ref_available(), reason="the reference build (oracle/_ref) is absent")
@pytest.mark.parametrize("seed", [1, 2])
def test_keep_mask_port_equals_reference(seed):
    q, nd, P, ref, alt, chrom, total = _random_case(seed)
    for maf, maxmiss, auto, mono, tv, strand in itertools.product(
            (0.0, 0.01, 0.05), (1.0, 0.5, 0.0), (0, 1), (0, 1), (0, 1), (0, 1, 2)):
        kw = dict(maf_min=maf, maxmiss=maxmiss, autosomes_only=auto, drop_monomorphic=mono,
                  transversions_only=tv, strand_mode=strand, total_indiv=total)
        kp, sp = oracle.keep_mask(q, nd, P, ref, alt, chrom, lib="port", **kw)
        kr, sr = oracle.keep_mask(q, nd, P, ref, alt, chrom, lib="ref", **kw)
        assert np.array_equal(kp, kr), kw
        assert np.array_equal(sp, sr), kw


def test_keep_mask_rules_by_hand():
    """Anchors: each rule drops exactly the SNPs it names."""
    P, M = 2, 6
    # SNP: 0 fine, 1 strand-ambiguous A/T, 2 multiallelic A/A, 3 transition A/G, 4 chrom 23,
    # 5 monomorphic
    ac2 = np.array([[2, 3], [2, 3], [2, 3], [2, 3], [2, 3], [0, 0]], np.int32)
    n = np.full((M, P), 4, np.int32)
    q, _, nd = oracle.counts_to_qvn(ac2.reshape(-1), n.reshape(-1))
    ref = ["A", "A", "A", "A", "C", "C"]
    alt = ["C", "T", "a", "G", "A", "A"]
    chrom = np.array([1, 1, 1, 1, 23, 1], np.int32)
    k, s = oracle.keep_mask(q, nd, P, ref, alt, chrom, strand_mode=0, total_indiv=4)
    assert k.tolist() == [1, 0, 0, 1, 1, 1]
    k, _ = oracle.keep_mask(q, nd, P, ref, alt, chrom, strand_mode=2, total_indiv=4)  # flip keeps, as keep
    assert k.tolist() == [1, 1, 0, 1, 1, 1]
    k, _ = oracle.keep_mask(q, nd, P, ref, alt, chrom, autosomes_only=True, drop_monomorphic=True,
                            transversions_only=True, total_indiv=4)
    assert k.tolist() == [1, 0, 0, 0, 0, 0]
    assert s[0, 0] == 5.0 / 16.0 and s[3, 0] == 8.0  # pooled ref AF (ac 2.5 of 8), allele count
