"""The fixed-point tensor-core arithmetic (precision "fixed_i8") against the FP64 oracle at
the headline population count, on blocks long enough to need more than one accumulator
segment, and its bounded-wait error path.

Tolerance (the same as test_gpu_parity.TOL["fixed_i8"]): |gpu - oracle| <= 1e-9 + 1e-6 *
|oracle| element-wise, relative 1e-6 with an absolute floor of 1e-9 (1e-6 of an f2 of 1e-3);
vpair, block sizes and the slab symmetry are exact.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from steppecu_b200 import F2Tensor, StpError, synth

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-9


def _oracle(rec, sel, po, block_id, n_block, pl):
    f2, vp, bs = oracle.f2_from_panel(rec, sel, po, block_id, n_block, pl, threads=16)
    return F2Tensor(f2, vp, bs, len(po) - 1, n_block)


def _check(got: F2Tensor, want: F2Tensor, rtol=RTOL, atol=ATOL):
    assert np.array_equal(got.block_sizes, want.block_sizes)
    assert np.array_equal(got.vpair, want.vpair), "vpair must be bit-exact"
    d = np.abs(got.f2 - want.f2)
    big = np.abs(want.f2) >= 1e-12
    rel = d[big] / np.abs(want.f2[big])
    print(f"max abs {d.max():.3e}  max rel(|f2|>=1e-12) {rel.max(initial=0):.3e}  "
          f"max comb(1e-9) {(d / (1e-9 + np.abs(want.f2))).max():.3e}  "
          f"max comb(1e-3) {(d / np.maximum(np.abs(want.f2), 1e-3)).max():.3e}")
    bad = d > atol + rtol * np.abs(want.f2)
    assert not bad.any(), (int(bad.sum()), float(d.max()))
    cube = got.cube()
    assert np.array_equal(cube, cube.transpose(1, 0, 2)), "f2 slabs must be exactly symmetric"


def _mixed_blocks(n_snp: int, sizes: list[int]) -> tuple[np.ndarray, int]:
    """A partition with the given leading block sizes, the rest in blocks of 700."""
    out, b, s = np.zeros(n_snp, np.int32), 0, 0
    for k in sizes:
        out[s:s + k] = b
        s += k
        b += 1
    while s < n_snp:
        k = min(700, n_snp - s)
        out[s:s + k] = b
        s += k
        b += 1
    return out, b


@pytest.fixture(scope="module")
def headline_shape():
    """1,000 populations x 10 samples (half pseudo-haploid, Beta(2,3) missingness) over 6,000
    SNPs: all 36 tile pairs of 8 row tiles, blocks from 1 to 2,500 SNPs in cost order, and
    population 3 missing at every SNP of block 2 (so its pairs there have vpair = 0)."""
    p = synth.generate("c3", seed=20261211, n_snp=6000)
    sel, po = p.selection()
    rec = p.records_numpy().copy()
    bid, nb = _mixed_blocks(p.n_snp, [1, 2500, 33, 1, 64, 65, 31, 1000, 2])
    s0, s1 = np.flatnonzero(bid == 2)[[0, -1]]
    for row in sel[po[3]:po[4]]:  # code 3 = missing (MSB-first, 4 codes per byte)
        byte, shift = row // 4, 6 - 2 * (row % 4)
        rec[s0:s1 + 1, byte] |= np.uint8(3 << shift)
    pl = oracle.detect_ploidy_pa(rec, sel)
    return rec, p.n_ind, sel, po, bid, nb, pl, _oracle(rec, sel, po, bid, nb, pl)


def test_fixed_i8_at_1000_populations_vs_oracle(ctx, headline_shape):
    rec, n_ind, sel, po, bid, nb, pl, want = headline_shape
    assert want.vpair.reshape(nb, 1000, 1000)[2, 3, :].max() == 0  # the all-missing pair is there
    got = ctx.extract_blocks(rec, n_ind, sel, po, bid, nb, precision="fixed_i8", sample_ploidy=pl)
    _check(got, want)


def test_split_f16_at_1000_populations_vs_oracle(ctx, headline_shape):
    """The split-F16 arithmetic at the same shape, at its own (wider) tolerance."""
    rec, n_ind, sel, po, bid, nb, pl, want = headline_shape
    got = ctx.extract_blocks(rec, n_ind, sel, po, bid, nb, precision="split_f16", sample_ploidy=pl)
    _check(got, want, rtol=5e-6, atol=2e-7)


@pytest.mark.parametrize("out_on_device", [False, True])
def test_fixed_i8_long_blocks_span_accumulator_segments(ctx, out_on_device):
    """Blocks of 16,384 SNPs and more: the int32 accumulators are read out every 16,384 SNPs
    and the block's sum continues in FP64."""
    import torch

    p = synth.generate("c2", seed=5, n_snp=40_000, n_pop=130)
    sel, po = p.selection()
    rec = p.records_numpy()
    bid, nb = _mixed_blocks(p.n_snp, [16_384, 16_385, 3, 7_228])
    pl = oracle.detect_ploidy_pa(rec, sel)
    want = _oracle(rec, sel, po, bid, nb, pl)
    if out_on_device:
        n = 130 * 130 * nb
        out = (torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.float64, device="cuda"))
        _, _, bs = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, nb, precision="fixed_i8", sample_ploidy=pl, out=out)
        got = F2Tensor(out[0].cpu().numpy(), out[1].cpu().numpy(), bs, 130, nb)
    else:
        got = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, nb, precision="fixed_i8", sample_ploidy=pl)
    _check(got, want)


def test_fixed_i8_block_longer_than_one_count_accumulation(ctx):
    """A block of 530,000 SNPs: the vpair kernel's int32 accumulator holds 524,032 SNPs of
    64 x 64 products, so the block's counts come from two accumulations (and its f2 from 33
    segments of 16,384 SNPs); a short block follows."""
    p = synth.generate("c1", seed=21, n_snp=531_000, n_pop=9)
    sel, po = p.selection()
    rec = p.records_numpy()
    bid = (np.arange(p.n_snp) >= 530_000).astype(np.int32)
    pl = oracle.detect_ploidy_pa(rec, sel)
    want = _oracle(rec, sel, po, bid, 2, pl)
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, 2, precision="fixed_i8", sample_ploidy=pl)
    assert want.vpair.max() > 524_032
    _check(got, want)


def test_fixed_i8_wait_timeout_reports_and_context_recovers():
    """A wait that runs out (the hook stops the f2 kernel's feed) ends the call with
    STP_DEVICE_TIMEOUT; the kernel frees its tensor memory and exits, and the same context
    then extracts correctly."""
    from steppecu_b200 import Context

    p = synth.generate("c1", seed=11, n_snp=3000, n_pop=9)
    sel, po = p.selection()
    rec = p.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel)
    want = _oracle(rec, sel, po, p.block_id, p.n_block, pl)
    with Context(0) as c:
        c.set_wait_bounds(timeout_ns=50_000_000, withhold_stage=0)
        with pytest.raises(StpError, match="device_timeout"):
            c.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8", sample_ploidy=pl)
        c.set_wait_bounds()
        for _ in range(2):
            got = c.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8",
                                   sample_ploidy=pl)
            _check(got, want)


@pytest.mark.parametrize("P", [41, 150, 250])
def test_tile_classes_do_not_change_results(ctx, P):
    """The partial-feed tile classes (stp_set_tile_classes) only change which rows a stage
    copies: every class mask gives the same f2 and vpair, bit for bit."""
    p = synth.generate("c4", seed=300 + P, n_snp=20_000, n_pop=P)
    sel, po = p.selection()
    rec = p.records_numpy()
    outs = []
    for mask in (0, 0xFFFF, 0x5555):
        ctx.set_tile_classes(mask)
        t = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8")
        outs.append(t)
    ctx.set_tile_classes(0x7FFF)
    for t in outs[1:]:
        assert np.array_equal(t.f2, outs[0].f2) and np.array_equal(t.vpair, outs[0].vpair)
