"""The CPU oracle pinned against the reference's own known-answer tests and, where the
reference's CpuBackend was built in place (oracle/_ref), against the reference itself.

Anchors restate the hand-computed cases of tests/unit/test_decode.cpp:274-298,
tests/unit/test_f2.cpp:123-134 and tests/unit/test_block_partition.cpp:53-202.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from steppecu_b200 import synth
from steppecu_b200.blocks import assign_blocks as py_assign_blocks


def pack_pa(codes: np.ndarray) -> np.ndarray:
    """codes [M, N] -> PA records [M, max(48, ceil(N/4))], MSB-first."""
    M, N = codes.shape
    bpr = max(48, (N + 3) // 4)
    out = np.zeros((M, bpr), np.uint8)
    for g in range(N):
        out[:, g // 4] |= (codes[:, g].astype(np.uint8) << (6 - 2 * (g % 4)))
    return out


# ---- decode (tests/unit/test_decode.cpp) ----------------------------------------------------

def test_genotype_code_positions_and_mod4():
    b = 0b11100100
    assert [oracle.genotype_code(b, k) for k in range(4)] == [3, 2, 1, 0]
    assert oracle.genotype_code(b, 4) == oracle.genotype_code(b, 0)
    assert oracle.genotype_code(b, 7) == oracle.genotype_code(b, 3)


def _counts(codes_per_sample, ploidies):
    codes = np.asarray(codes_per_sample, np.uint8)[None, :]
    rec = pack_pa(codes)
    sel = np.arange(codes.shape[1], dtype=np.int64)
    ac2, n = oracle.decode_counts_pa(rec, sel, [0, codes.shape[1]], np.asarray(ploidies, np.int32))
    return int(ac2[0]) / 2.0, int(n[0])


@pytest.mark.parametrize("codes,ploidies,ac,n", [
    ([0, 1, 2, 3], [2, 2, 2, 2], 3.0, 6),      # diploid == legacy fold: ac=3, n=2*3
    ([0, 2, 2, 3], [1, 1, 1, 1], 2.0, 3),      # pseudo-haploid homozygous: code/2, n += 1
    ([2, 1], [1, 1], 1.5, 2),                  # PH out-of-window het adds +0.5
    ([3, 3], [2, 1], 0.0, 0),                  # missing excluded regardless of ploidy
    ([2, 2, 2], [0, 3, -1], 0.0, 0),           # bad ploidy contributes nothing
    ([1, 2], [2, 1], 2.0, 3),                  # mixed-ploidy pop: 1/(3-2) + 2/(3-1)
    ([2, 2, 3, 1], [2, 2, 2, 2], 5.0, 6),      # accumulate then finalize: q = 5/6
])
def test_decode_fold_anchors(codes, ploidies, ac, n):
    got_ac, got_n = _counts(codes, ploidies)
    assert (got_ac, got_n) == (ac, n)
    q, v, nd = oracle.counts_to_qvn(np.array([int(2 * ac)], np.int32), np.array([n], np.int32))
    if n > 0:
        assert v[0] == 1.0 and nd[0] == float(n) and q[0] == ac / n
    else:
        assert q[0] == 0.0 and v[0] == 0.0 and nd[0] == 0.0


def test_finalize_single_pseudohaploid():
    q, v, nd = oracle.counts_to_qvn(np.array([2], np.int32), np.array([1], np.int32))
    assert (q[0], v[0], nd[0]) == (1.0, 1.0, 1.0)


def test_detect_ploidy_window():
    # Sample 0: het at SNP 5 -> diploid. Sample 1: het only after SNP 1000 -> pseudo-haploid.
    M = 1200
    codes = np.zeros((M, 3), np.uint8)
    codes[5, 0] = 1
    codes[1100, 1] = 1
    codes[:, 2] = 2
    rec = pack_pa(codes)
    sel = np.arange(3, dtype=np.int64)
    assert list(oracle.detect_ploidy_pa(rec, sel)) == [2, 1, 1]
    canon, obpr = oracle.transpose_pa_to_canonical(rec, sel)
    assert list(oracle.detect_ploidy_canonical(canon, obpr, M, 3)) == [2, 1, 1]


# ---- f2 (tests/unit/test_f2.cpp) ---------------------------------------------------------------

def _f2_one(q, n, v=None):
    q = np.asarray(q, np.float64)
    P, M = q.shape
    v = np.ones_like(q) if v is None else np.asarray(v, np.float64)
    n = np.asarray(n, np.float64)
    flat = lambda a: np.ascontiguousarray(a.T).ravel()  # column-major [P x M]
    f2, vp, bs = oracle.compute_f2_blocks(flat(q), flat(v), flat(n), P, np.zeros(M, np.int32), 1)
    return f2.reshape(P, P, order="F"), vp.reshape(P, P, order="F")


def test_f2_term_anchor():
    # h_i = 0.7*0.3/21 = 0.01, h_j = 0.2*0.8/8 = 0.02: term = 0.5^2 - 0.03 = 0.22
    f2, vp = _f2_one([[0.7], [0.2]], [[22.0], [9.0]])
    assert abs(f2[0, 1] - 0.22) <= 1e-12 and f2[1, 0] == f2[0, 1] and vp[0, 1] == 1.0


def test_het_denominator_floor_and_diagonal():
    # n = 1 -> max(n-1, 1) = 1: h = 0.25; the diagonal keeps -2*mean(h) (not zero).
    f2, _ = _f2_one([[0.5]], [[1.0]])
    assert abs(f2[0, 0] - (-0.5)) <= 1e-15


def test_vpair_zero_guard():
    f2, vp = _f2_one([[0.5], [0.3]], [[4.0], [4.0]], v=[[1.0], [0.0]])
    assert f2[0, 1] == 0.0 and vp[0, 1] == 0.0


def test_assemble_matches_term_sum():
    pi, pj = np.array([0.7, 0.3, 0.9]), np.array([0.2, 0.5, 0.1])
    ni, nj = np.array([10.0, 20.0, 30.0]), np.array([8.0, 12.0, 40.0])
    f2, _ = _f2_one([pi, pj], [ni, nj])
    hi = pi * (1 - pi) / (ni - 1)
    hj = pj * (1 - pj) / (nj - 1)
    want = np.mean((pi - pj) ** 2 - hi - hj)
    assert abs(f2[0, 1] - want) <= 1e-12


def test_malformed_partition_raises():
    q = np.full(4 * 2, 0.5)
    with pytest.raises(ValueError):
        oracle.compute_f2_blocks(q, np.ones(8), np.full(8, 4.0), 2, np.array([0, 1, 0, 1], np.int32), 2)


def test_degenerate_extents_give_zeros():
    f2, vp, bs = oracle.compute_f2_blocks(np.zeros(0), np.zeros(0), np.zeros(0), 3, np.zeros(0, np.int32), 2)
    assert f2.shape == (18,) and not f2.any() and not vp.any() and not bs.any()


# ---- block walk (tests/unit/test_block_partition.cpp) -------------------------------------

BLOCK_CASES = [
    ([1, 1, 1, 1], [0.0, 0.01, 0.02, 0.049], [0, 0, 0, 0]),
    ([1, 1, 1], [0.00, 0.05, 0.10], [0, 1, 2]),                        # inclusive >= cut
    ([1, 1, 1, 1], [0.00, 0.04, 0.06, 0.10], [0, 0, 1, 1]),             # re-anchor, remainder rolls forward
    ([1, 1, 2, 2], [0.00, 0.01, 0.00, 0.02], [0, 0, 1, 1]),             # chromosome change
    ([7, 7, 7, 7, 7], [0.0] * 5, [0] * 5),                              # all-zero chromosome
    ([16, 17, 17, 17], [1.340230, -0.000258, -0.000238, 0.000249], [0, 1, 1, 1]),
    ([1, 1, 1], [0.01, 0.06, 0.16], [0, 0, 1]),                          # FP knife edge: 0.06-0.01 < 0.05
]


@pytest.mark.parametrize("chrom,gp,want", BLOCK_CASES)
def test_block_walk_anchors(chrom, gp, want):
    bid, nb = oracle.assign_blocks(chrom, gp, 0.05)
    assert list(bid) == want and nb == max(want) + 1
    pid, pnb = py_assign_blocks(chrom, gp, 0.05)
    assert list(pid) == want and pnb == nb


@pytest.mark.parametrize("width", [0.0, -0.05, float("nan")])
def test_block_walk_illegal_width(width):
    assert oracle.assign_blocks([1, 1, 1], [0.0, 0.06, 0.12], width)[1] == 0
    assert py_assign_blocks([1, 1, 1], [0.0, 0.06, 0.12], width)[1] == 0


def test_block_walk_bp_fallback():
    chrom = [1] * 5
    gp = [0.0] * 5
    pp = [1.0, 1.5e6, 2.1e6, 3.0e6, 4.2e6]
    bid, nb = oracle.assign_blocks(chrom, gp, 0.05, pp)
    pid, pnb = py_assign_blocks(chrom, gp, 0.05, pp)
    assert list(bid) == [0, 0, 1, 1, 2] and list(pid) == list(bid) and nb == pnb == 3


def test_block_walk_matches_port_on_panel():
    p = synth.generate("c1", seed=3, n_snp=20000, n_pop=4)
    bid, nb = oracle.assign_blocks(p.chrom, p.genpos, 0.05, p.physpos)
    assert nb == p.n_block and np.array_equal(bid, p.block_id)


# ---- the port against the reference's own CpuBackend --------------------------------------

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference CpuBackend not built (oracle/_ref)")


@pytest.fixture(scope="module")
def small_panel():
    p = synth.generate("c1", seed=11, n_snp=3000, n_pop=6)
    sel, po = p.selection()
    return p, sel, po


@needs_ref
def test_port_decode_af_equals_reference(small_panel):
    p, sel, po = small_panel
    rec = p.records_numpy()
    canon, obpr = oracle.transpose_pa_to_canonical(rec, sel)
    for detect in (True, False):
        a = oracle.decode_af_canonical(canon, obpr, p.n_snp, po, detect=detect)
        b = oracle.decode_af_canonical(canon, obpr, p.n_snp, po, detect=detect, lib="ref")
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@needs_ref
def test_port_counts_match_reference_decode(small_panel):
    """The integer decode (ac2, n) of SNP-major records reproduces the reference's FP64
    decode_af of the canonical tile exactly."""
    p, sel, po = small_panel
    rec = p.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = oracle.decode_counts_pa(rec, sel, po, pl)
    q, v, nd = oracle.counts_to_qvn(ac2, n)
    canon, obpr = oracle.transpose_pa_to_canonical(rec, sel)
    rq, rv, rn = oracle.decode_af_canonical(canon, obpr, p.n_snp, po, detect=True, lib="ref")
    assert np.array_equal(q, rq) and np.array_equal(v, rv) and np.array_equal(nd, rn)


@needs_ref
def test_port_f2_blocks_equal_reference(small_panel):
    p, sel, po = small_panel
    rec = p.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = oracle.decode_counts_pa(rec, sel, po, pl)
    q, v, nd = oracle.counts_to_qvn(ac2, n)
    a = oracle.compute_f2_blocks(q, v, nd, p.n_pop, p.block_id, p.n_block)
    b = oracle.compute_f2_blocks(q, v, nd, p.n_pop, p.block_id, p.n_block, lib="ref")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    c = oracle.compute_f2_blocks_sharded(q, v, nd, p.n_pop, p.block_id, p.n_block, threads=3, lib="ref")
    for x, y in zip(a, c):
        assert np.array_equal(x, y)


@needs_ref
def test_port_block_walk_equals_reference():
    p = synth.generate("c1", seed=5, n_snp=8000, n_pop=2)
    a = oracle.assign_blocks(p.chrom, p.genpos, 0.05, p.physpos)
    b = oracle.assign_blocks(p.chrom, p.genpos, 0.05, p.physpos, lib="ref")
    assert a[1] == b[1] and np.array_equal(a[0], b[0])


@needs_ref
def test_port_jackknife_equals_reference():
    rng = np.random.default_rng(2)
    m, nb = 7, 30
    x = rng.normal(0.02, 0.01, size=m * nb)
    bs = rng.integers(50, 4000, size=nb).astype(np.int32)
    e1, v1 = oracle.block_jackknife(x, bs, m, nb)
    e2, v2 = oracle.block_jackknife(x, bs, m, nb, lib="ref")
    np.testing.assert_allclose(e1, e2, rtol=1e-14, atol=0)
    np.testing.assert_allclose(v1, v2, rtol=1e-12, atol=0)
