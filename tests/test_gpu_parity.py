"""GPU parity through the C ABI against the CPU oracle on identical seeded inputs.

Counts, ploidy, vpair and the canonical decode are compared bit for bit. f2 is compared
with the tolerance of each contraction arithmetic (see TOL), checked as
|gpu - oracle| <= atol + rtol * |oracle| element-wise, with the worst errors printed.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import steppecu_b200 as sb
from steppecu_b200 import F2Tensor, StpError, extract_f2, read_f2, synth
from steppecu_b200.synth import write_eigenstrat

pytestmark = pytest.mark.gpu

# Per-arithmetic f2 tolerance (rtol, atol) against the FP64 oracle. The floating forms sum
# the numerator in FP32 over short SNP chunks and combine chunks in FP64. Split-F16 keeps
# ~22 mantissa bits per operand and FP32 SIMT 24; split-BF16 (hi+lo) keeps only ~16, so its
# per-element error is ~2^-17 and its tolerance is wider. The fixed-point form sums exactly
# in integers over 32-bit fixed-point operands: relative 1e-6 with an absolute floor of
# 1e-9, i.e. |gpu - oracle| <= 1e-6 * max(|oracle|, 1e-3) up to a factor of two. The floor
# is 1e-6 of an f2 of 1e-3, an order of magnitude below the per-block f2 values and their
# sampling spread on these panels, and it is where a relative bound stops meaning anything
# (f2 estimates cross zero).
TOL = {
    "fp32": (5e-6, 5e-8),
    "split_f16": (5e-6, 2e-7),
    "split_f16_fine": (5e-6, 2e-7),
    "split_bf16": (3e-4, 3e-6),
    "fixed_i8": (1e-6, 1e-9),
}
MODES = ["fp32", "split_bf16", "split_f16", "split_f16_fine", "fixed_i8"]
TC_DEFAULT = "fixed_i8"


def oracle_f2(panel, sel, po, ploidy=None, block_id=None, n_block=None):
    rec = panel.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel) if ploidy is None else ploidy
    bid = panel.block_id if block_id is None else block_id
    nb = panel.n_block if n_block is None else n_block
    f2, vp, bs = oracle.f2_from_panel(rec, sel, po, bid, nb, pl, threads=8)
    return F2Tensor(f2, vp, bs, len(po) - 1, nb), pl


def f2_error(got: np.ndarray, want: np.ndarray) -> dict:
    d = np.abs(got - want)
    rel = d / np.maximum(np.abs(want), 1e-300)
    big = np.abs(want) >= 1e-12
    return {"max_abs": float(d.max(initial=0)), "max_rel": float(rel[big].max(initial=0)),
            "max_comb": float((d / (1e-9 + np.abs(want))).max(initial=0))}


def assert_f2_close(got: F2Tensor, want: F2Tensor, mode: str):
    assert got.P == want.P and got.n_block == want.n_block
    assert np.array_equal(got.block_sizes, want.block_sizes)
    assert np.array_equal(got.vpair, want.vpair), "vpair must be bit-exact"
    rtol, atol = TOL[mode]
    err = f2_error(got.f2, want.f2)
    print(f"[{mode}] f2 error vs oracle: {err}")
    bad = np.abs(got.f2 - want.f2) > atol + rtol * np.abs(want.f2)
    assert not bad.any(), (err, int(bad.sum()))
    cube = got.cube()
    assert np.array_equal(cube, cube.transpose(1, 0, 2)), "f2 slabs must be exactly symmetric"


@pytest.fixture(scope="module")
def c1():
    p = synth.generate("c1", seed=20261203)
    sel, po = p.selection()
    want, pl = oracle_f2(p, sel, po)
    return p, sel, po, want, pl


@pytest.fixture(scope="module")
def uneven():
    """Uneven population sizes (1..60), half pseudo-haploid, Beta(2,3) missingness,
    lognormal blocks: the shape of the batched-uneven workload at test size."""
    p = synth.generate("c4", seed=7, n_snp=40_000, n_pop=37)
    sel, po = p.selection()
    want, pl = oracle_f2(p, sel, po)
    return p, sel, po, want, pl


# ---- decode -------------------------------------------------------------------------------

def test_detect_ploidy_bitexact(ctx, uneven):
    p, sel, po, _, pl = uneven
    got = ctx.detect_ploidy(p.records_numpy(), p.n_ind, sel)
    assert np.array_equal(got, pl)
    # The generator's truth: every diploid with a het in the window is found.
    assert set(np.unique(got)) <= {1, 2}


@pytest.mark.parametrize("ploidy", ["auto", "pseudo", "diploid"])
def test_decode_counts_bitexact(ctx, uneven, ploidy):
    p, sel, po, _, pl = uneven
    rec = p.records_numpy()
    if ploidy == "auto":
        opl = pl
    else:
        opl = np.full(sel.size, 1 if ploidy == "pseudo" else 2, np.int32)
    ac2, n = ctx.decode_counts(rec, p.n_ind, sel, po, ploidy=ploidy)
    wa, wn = oracle.decode_counts_pa(rec, sel, po, opl)
    P = len(po) - 1
    assert np.array_equal(ac2, wa.reshape(-1, P).T) and np.array_equal(n, wn.reshape(-1, P).T)


def test_decode_counts_device_records(ctx, uneven):
    import torch

    p, sel, po, _, pl = uneven
    rec = p.records_numpy()
    d = torch.as_tensor(rec).cuda()
    ac2, n = ctx.decode_counts(d, p.n_ind, sel, po, sample_ploidy=pl)
    wa, wn = oracle.decode_counts_pa(rec, sel, po, pl)
    P = len(po) - 1
    assert np.array_equal(ac2, wa.reshape(-1, P).T) and np.array_equal(n, wn.reshape(-1, P).T)


@pytest.mark.parametrize("panel_pops,n_snp", [(1232, 4001), (1250, 4000)])
def test_wide_panel_scattered_selection(ctx, panel_pops, n_snp):
    """40 scattered populations, in descending order, from panels of 12,320 and 12,500
    samples. 12,320 samples give 3,080-byte records, a multiple of 4 bytes but not of 16,
    which the transpose reads at their own pitch with 4-byte copies; 12,500 samples give
    3,125-byte records, which are re-pitched to 16 bytes first. Counts bit-exact, f2 within
    tolerance."""
    p = synth.generate("c3", seed=panel_pops + n_snp, n_snp=n_snp, n_pop=panel_pops)
    sel, po = p.selection(list(range(panel_pops - 1, -1, -31))[:40])
    rec = p.records_numpy()
    P = len(po) - 1
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = ctx.decode_counts(rec, p.n_ind, sel, po)
    wa, wn = oracle.decode_counts_pa(rec, sel, po, pl)
    assert np.array_equal(ac2, wa.reshape(-1, P).T) and np.array_equal(n, wn.reshape(-1, P).T)
    want, _ = oracle_f2(p, sel, po, ploidy=pl)
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=TC_DEFAULT)
    assert_f2_close(got, want, TC_DEFAULT)


@pytest.mark.parametrize("size,n_pop,n_snp", [(250, 5, 3000), (16383, 1, 300)])
def test_decode_counts_large_populations(ctx, size, n_pop, n_snp):
    """Populations far above the decode's in-register sample window, up to the largest
    population the 16-bit count packing admits (ac2 <= 2 * 16383)."""
    import dataclasses

    wl = dataclasses.replace(synth.WORKLOADS["c2"], name="large", n_pop=n_pop, ind_per_pop=size)
    p = synth.generate(wl, seed=size, n_snp=n_snp)
    sel, po = p.selection()
    rec = p.records_numpy()
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = ctx.decode_counts(rec, p.n_ind, sel, po)
    wa, wn = oracle.decode_counts_pa(rec, sel, po, pl)
    assert np.array_equal(ac2, wa.reshape(-1, n_pop).T) and np.array_equal(n, wn.reshape(-1, n_pop).T)
    if n_pop > 1:
        want, _ = oracle_f2(p, sel, po)
        got = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=TC_DEFAULT)
        assert_f2_close(got, want, TC_DEFAULT)


def test_detect_ploidy_tile_bitexact(ctx, uneven):
    p, sel, _, _, _ = uneven
    canon, obpr = oracle.transpose_pa_to_canonical(p.records_numpy()[:3000], sel)
    got = ctx.detect_ploidy_tile(canon, obpr, 3000)
    want = oracle.detect_ploidy_canonical(canon, obpr, 3000, sel.size)
    assert np.array_equal(got, want) and set(np.unique(got)) <= {1, 2}


@pytest.mark.parametrize("detect", [True, False])
def test_decode_af_canonical_bitexact(ctx, uneven, detect):
    p, sel, po, _, _ = uneven
    canon, obpr = oracle.transpose_pa_to_canonical(p.records_numpy()[:5000], sel)
    got = ctx.decode_af(canon, obpr, 5000, po, ploidy=2, detect=detect)
    want = oracle.decode_af_canonical(canon, obpr, 5000, po, ploidy=2, detect=detect)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


# ---- f2 ------------------------------------------------------------------------------------

@pytest.mark.parametrize("mode", MODES)
def test_f2_c1_vs_oracle(ctx, c1, mode):
    p, sel, po, want, pl = c1
    got = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    assert_f2_close(got, want, mode)


@pytest.mark.parametrize("mode", MODES)
def test_f2_uneven_vs_oracle(ctx, uneven, mode):
    p, sel, po, want, pl = uneven
    got, used = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, p.n_block, precision=mode,
                                   return_ploidy=True)
    assert np.array_equal(used, pl)
    assert_f2_close(got, want, mode)


@pytest.mark.parametrize("mode", MODES)
def test_f2_from_qvn_vs_oracle(ctx, c1, mode):
    p, sel, po, want, pl = c1
    ac2, n = oracle.decode_counts_pa(p.records_numpy(), sel, po, pl)
    q, v, nd = oracle.counts_to_qvn(ac2, n)
    got = ctx.f2_from_qvn(q, v, nd, p.n_pop, p.block_id, p.n_block, precision=mode)
    assert_f2_close(got, want, mode)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("P", [1, 2, 7, 65, 130])
def test_f2_odd_population_counts(ctx, mode, P):
    p = synth.generate("c4", seed=100 + P, n_snp=6000, n_pop=P)
    sel, po = p.selection()
    want, _ = oracle_f2(p, sel, po)
    got = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    assert_f2_close(got, want, mode)


@pytest.mark.parametrize("mode", MODES)
def test_f2_edge_blocks_and_missing(ctx, mode):
    """Blocks of one SNP, an empty block id, and a population whose samples are all
    missing in one block (vpair = 0 -> f2 = 0)."""
    p = synth.generate("c1", seed=9, n_snp=3000, n_pop=5)
    rec = p.records_numpy().copy()
    sel, po = p.selection()
    # population 2 entirely missing in SNPs [100, 400)
    for g in sel[po[2]:po[3]]:
        rec[100:400, g // 4] |= np.uint8(3 << (6 - 2 * (g % 4)))
    bid = np.zeros(3000, np.int32)
    bid[1:2] = 1            # block 1: one SNP
    bid[2:100] = 2
    bid[100:400] = 4        # block 3 left empty
    bid[400:] = 5
    nb = 6
    pl = oracle.detect_ploidy_pa(rec, sel)
    f2, vp, bs = oracle.f2_from_panel(rec, sel, po, bid, nb, pl)
    want = F2Tensor(f2, vp, bs, 5, nb)
    got = ctx.extract_blocks(rec, p.n_ind, sel, po, bid, nb, precision=mode)
    assert list(got.block_sizes) == [1, 1, 98, 0, 300, 2600]
    assert not got.f2[25 * 3:25 * 4].any() and not got.vpair[25 * 3:25 * 4].any()
    assert got.vpair[2 + 5 * 0 + 25 * 4] == 0.0 and got.f2[2 + 5 * 0 + 25 * 4] == 0.0
    assert_f2_close(got, want, mode)


def test_f2_deterministic(ctx, c1):
    p, sel, po, _, _ = c1
    a = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, p.n_block, precision=MODES[-1])
    b = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, p.n_block, precision=MODES[-1])
    assert np.array_equal(a.f2, b.f2) and np.array_equal(a.vpair, b.vpair)


def test_degenerate_requests(ctx):
    p = synth.generate("c1", seed=1, n_snp=500, n_pop=3)
    sel, po = p.selection()
    t = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, 0)
    assert t.f2.size == 0
    z = ctx.extract_blocks(p.records_numpy()[:0], p.n_ind, sel, po, np.zeros(0, np.int32), 2)
    assert z.f2.shape == (18,) and not z.f2.any() and not z.vpair.any() and list(z.block_sizes) == [0, 0]


def test_malformed_partition_is_an_error(ctx):
    p = synth.generate("c1", seed=1, n_snp=500, n_pop=3)
    sel, po = p.selection()
    bad = p.block_id.copy()
    bad[10] = bad[-1] + 5
    with pytest.raises(StpError, match="runtime_error"):
        ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, bad, p.n_block)
    with pytest.raises(StpError, match="invalid_argument"):
        ctx.extract_blocks(p.records_numpy(), p.n_ind, np.array([p.n_ind + 3]), [0, 1], p.block_id, p.n_block)


def test_plan_device_resident_matches_one_shot(ctx, c1):
    import torch

    p, sel, po, want, _ = c1
    rec = torch.as_tensor(p.records_numpy()).cuda()
    plan = ctx.plan(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=MODES[-1])
    n = p.n_pop ** 2 * p.n_block
    f2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    vp = torch.zeros_like(f2)
    for _ in range(2):
        plan.run(rec, f2, vp, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    one = ctx.extract_blocks(p.records_numpy(), p.n_ind, sel, po, p.block_id, p.n_block, precision=MODES[-1])
    assert np.array_equal(f2.cpu().numpy(), one.f2) and np.array_equal(vp.cpu().numpy(), one.vpair)
    assert plan.launches >= 2


def test_closing_the_context_closes_its_plans(c1):
    """A plan still open when its context closes is destroyed first (it uses the context's
    stream and workspaces); running it afterwards is refused on the host, and so is a new
    plan on the closed context."""
    import torch

    p, sel, po, _, _ = c1
    rec = torch.as_tensor(p.records_numpy()).cuda()
    c = sb.Context(0)
    plan = c.plan(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8")
    c.close()
    assert plan._h is None
    f2 = torch.zeros(p.n_pop ** 2 * p.n_block, dtype=torch.float64, device="cuda")
    with pytest.raises(StpError, match="invalid_argument"):
        plan.run(rec, f2, torch.zeros_like(f2))
    del plan
    with pytest.raises(ValueError, match="closed"):
        c.plan(rec, p.n_ind, sel, po, p.block_id, p.n_block)


@pytest.mark.parametrize("mode", [TC_DEFAULT, "fixed_i8"])
def test_plan_graph_replay_equals_plan_run(ctx, c1, mode):
    import torch

    p, sel, po, _, _ = c1
    rec = torch.as_tensor(p.records_numpy()).cuda()
    plan = ctx.plan(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    n = p.n_pop * p.n_pop * p.n_block
    f_a, v_a = torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.float64, device="cuda")
    plan.run(rec, f_a, v_a)
    torch.cuda.synchronize()
    f_b, v_b = torch.full_like(f_a, 7.0), torch.full_like(v_a, 7.0)
    before = ctx.launches
    for _ in range(3):  # the first call captures, the others replay
        f_b.fill_(7.0)
        v_b.fill_(7.0)
        plan.run_graph(rec, f_b, v_b)
    torch.cuda.synchronize()
    assert ctx.launches - before == 3 * plan.launches
    assert torch.equal(f_a, f_b) and torch.equal(v_a, v_b)
    plan.close()


@pytest.mark.parametrize("mode", [TC_DEFAULT, "fixed_i8"])
def test_per_block_launches_equal_persistent_launch(ctx, uneven, mode):
    import torch

    p, sel, po, _, _ = uneven
    rec = torch.as_tensor(p.records_numpy()).cuda()
    plan = ctx.plan(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    n = p.n_pop * p.n_pop * p.n_block
    out = [torch.full((n,), 3.0, dtype=torch.float64, device="cuda") for _ in range(4)]
    plan.run(rec, out[0], out[1])
    plan.set_per_block_launch(True)
    before = ctx.launches
    plan.run(rec, out[2], out[3])
    torch.cuda.synchronize()
    per_contraction = 2 if mode == "fixed_i8" else 1  # fixed point: the vpair kernel, then f2
    assert ctx.launches - before == plan.launches == 3 + per_contraction * p.n_block
    assert torch.equal(out[0], out[2]) and torch.equal(out[1], out[3])
    plan.close()


def test_jackknife_vs_oracle(ctx, c1):
    _, _, _, want, _ = c1
    m = want.P * want.P
    est, var = ctx.jackknife(want.f2, want.block_sizes, m, want.n_block)
    e2, v2 = oracle.block_jackknife(want.f2, want.block_sizes, m, want.n_block)
    np.testing.assert_allclose(est, e2, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(var, v2, rtol=1e-9, atol=1e-18)


def test_extract_f2_files_roundtrip(tmp_path, c1):
    p, sel, po, want, pl = c1
    write_eigenstrat(p, tmp_path / "panel")
    pops = list(reversed(p.pop_labels))  # P axis is sorted by label regardless of the order given
    out = extract_f2(tmp_path / "panel", pops=pops, out=str(tmp_path / "f2dir"), maxmiss=1.0,
                     precision=MODES[-1])
    h = read_f2(out)
    assert h.pops == sorted(p.pop_labels) and h.P == p.n_pop and h.n_block == p.n_block
    assert_f2_close(h.tensor, want, MODES[-1])
    h2 = extract_f2(tmp_path / "panel", pops=pops, maxmiss=1.0, precision=MODES[-1])
    assert np.array_equal(h2.to_numpy(), h.to_numpy())


def test_int_max_and_device_oom_statuses(ctx):
    """The reference's M > INT_MAX guard (std::runtime_error) and its device-OOM status
    (CudaError(cudaErrorMemoryAllocation) -> Status::DeviceOom), through the raw C ABI with
    tiny buffers that neither call reads: n_snp = 2^31 fails with STP_RUNTIME_ERROR before
    anything is allocated; 2^30 SNPs of 256-byte host records fail with STP_DEVICE_OOM when
    the 256 GiB upload buffer cannot be allocated. The context stays usable."""
    import ctypes as C

    from steppecu_b200 import _lib as L

    rec = np.zeros(256, np.uint8)
    sel = np.arange(4, dtype=np.int64)
    po = np.array([0, 2, 4], np.int64)
    bid = np.zeros(4, np.int32)
    f2, vp, bs = np.zeros(8), np.zeros(8), np.zeros(2, np.int32)

    def call(n_snp):
        g = L.GenoView(rec.ctypes.data, 256, 256, n_snp, 1024, 0)
        r = L.F2Request(g, sel.ctypes.data, po.ctypes.data, 2, None, L.PLOIDY_AUTO, bid.ctypes.data, 2,
                        L.PREC_SPLIT_F16)
        o = L.F2Output(f2.ctypes.data, vp.ctypes.data, bs.ctypes.data, 0, None)
        return L.lib().stp_f2_extract_blocks(ctx._h, C.byref(r), C.byref(o))

    assert call(2**31) == L.STP_RUNTIME_ERROR
    assert b"INT_MAX" in L.lib().stp_last_error()
    assert call(2**30) == L.STP_DEVICE_OOM
    p = synth.generate("c1", seed=3, n_snp=2000, n_pop=4)
    s2, po2 = p.selection()
    t = ctx.extract_blocks(p.records_numpy(), p.n_ind, s2, po2, p.block_id, p.n_block, precision=TC_DEFAULT)
    assert t.f2.size == 16 * p.n_block


@pytest.mark.parametrize("n_pop,misalign,wide", [(600, False, False), (603, False, False), (600, True, False),
                                                  (130, False, True)])
def test_host_output_equals_device_output(n_pop, misalign, wide):
    """Host outputs receive every f2 slab whole and the vpair slabs as packed upper tiles of
    16-bit counts (32-bit when a block has 65,536 SNPs or more), which the library widens
    into both halves of each slab on the host: with AVX2 streaming stores when P % 4 == 0 and
    the output is 32-byte aligned, else element by element (P = 603, and an output that
    starts 8 bytes past an aligned address). Each equals the device-output extraction bit
    for bit."""
    import torch

    from steppecu_b200 import Context

    p = synth.generate("c3", seed=n_pop, n_snp=70_000 if wide else 6_000, n_pop=n_pop)
    if wide:  # one block of 66,000 SNPs, then one of 4,000
        p.block_id = (np.arange(p.n_snp) >= 66_000).astype(np.int32)
        p.n_block = 2
    sel, po = p.selection()
    rec = p.records_numpy()
    P, B = p.n_pop, p.n_block
    n = P * P * B
    if misalign:  # both outputs start 8 bytes past a 32-byte boundary
        def at8(m):
            buf = np.zeros(m + 4)
            off = ((8 - buf.ctypes.data) % 32) // 8
            return buf[off:off + m]

        f2h, vph = at8(n), at8(n)
        assert f2h.ctypes.data % 32 == 8 and vph.ctypes.data % 32 == 8
    else:
        f2h, vph = np.zeros(n), np.zeros(n)
    f2d = torch.zeros(n, dtype=torch.float64, device="cuda")
    vpd = torch.zeros_like(f2d)
    for mode in ("fixed_i8", "split_f16"):
        with Context(0) as c:
            c.extract_blocks(rec, p.n_ind, sel, po, p.block_id, B, precision=mode, out=(f2h, vph))
            c.extract_blocks(torch.from_numpy(rec).cuda(), p.n_ind, sel, po, p.block_id, B, precision=mode,
                             out=(f2d, vpd))
        assert np.array_equal(f2h, f2d.cpu().numpy())
        assert np.array_equal(vph, vpd.cpu().numpy())
    if wide:
        assert vph.max() > 65535


def test_host_streaming_bounds_device_output_memory():
    """Host records and host outputs stream in segments of whole blocks through a two-segment
    ring of device slabs: the result equals the device-output extraction bit for bit, and the
    device memory the call takes stays well below the F2BlockTensor it returns."""
    import torch

    from steppecu_b200 import Context

    p = synth.generate("c3", seed=5, n_snp=20_000, n_pop=600)
    sel, po = p.selection()
    rec = p.records_numpy()
    P, B = p.n_pop, p.n_block
    full = 2 * P * P * B * 8
    with Context(0) as c:
        free0 = torch.cuda.mem_get_info(0)[0]
        t = c.extract_blocks(rec, p.n_ind, sel, po, p.block_id, B, precision="split_f16")
        taken = free0 - torch.cuda.mem_get_info(0)[0]
    assert taken < 0.5 * full, (taken, full)
    f2d = torch.zeros(P * P * B, dtype=torch.float64, device="cuda")
    vpd = torch.zeros_like(f2d)
    with Context(0) as c:
        c.extract_blocks(torch.from_numpy(rec).cuda(), p.n_ind, sel, po, p.block_id, B, precision="split_f16",
                         out=(f2d, vpd))
    assert np.array_equal(t.f2, f2d.cpu().numpy())
    assert np.array_equal(t.vpair, vpd.cpu().numpy())
