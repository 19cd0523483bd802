"""The streamed output tiers (stp_f2_extract_streamed, stp_f2_from_qvn_streamed: runs of
finished blocks handed to a callback, as compute_f2_blocks_streamed's StreamTarget), the
device-resident output from Q / V / N (stp_f2_from_qvn_device, as compute_f2_blocks_device),
and the disk tier of extract_f2, each bit for bit against the one-shot result."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from steppecu_b200 import StpError, extract_f2, read_f2, synth
from steppecu_b200.synth import write_eigenstrat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def panel():
    p = synth.generate("c2", seed=41, n_snp=60_000, n_pop=150)
    sel, po = p.selection()
    return p, sel, po, p.records_numpy()


def _collect(P, nb):
    f2 = np.full(P * P * nb, np.nan)
    vp = np.full(P * P * nb, np.nan)
    runs = []

    def sink(b0, b1, a, v):
        f2[b0 * P * P:b1 * P * P] = a
        vp[b0 * P * P:b1 * P * P] = v
        runs.append((b0, b1))

    return f2, vp, runs, sink


@pytest.mark.parametrize("mode", ["fixed_i8", "split_f16"])
@pytest.mark.parametrize("on_device", [False, True])
def test_streamed_extraction_equals_one_shot(ctx, panel, mode, on_device):
    import torch

    p, sel, po, rec = panel
    want = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision=mode)
    f2, vp, runs, sink = _collect(p.n_pop, p.n_block)
    src = rec
    if on_device:  # device records at a 16-byte pitch (the streamed path reads them in place)
        pitch = (rec.shape[1] + 15) // 16 * 16
        src = torch.zeros((rec.shape[0], pitch), dtype=torch.uint8, device="cuda")
        src[:, :rec.shape[1]] = torch.as_tensor(rec).cuda()
    bs = ctx.extract_streamed(src, p.n_ind, sel, po, p.block_id, p.n_block, sink, precision=mode)
    assert len(runs) > 2 and runs[0][0] == 0 and runs[-1][1] == p.n_block
    assert all(a[1] == b[0] for a, b in zip(runs, runs[1:]))  # in block order, contiguous
    assert np.array_equal(bs, want.block_sizes)
    assert np.array_equal(f2, want.f2) and np.array_equal(vp, want.vpair)


def test_from_qvn_streamed_and_device_equal_host(ctx, panel):
    import torch

    p, sel, po, rec = panel
    pl = oracle.detect_ploidy_pa(rec, sel)
    ac2, n = oracle.decode_counts_pa(rec, sel, po, pl)
    q, v, nd = oracle.counts_to_qvn(ac2, n)
    want = ctx.f2_from_qvn(q, v, nd, p.n_pop, p.block_id, p.n_block, precision="fixed_i8")
    f2, vp, _, sink = _collect(p.n_pop, p.n_block)
    bs = ctx.f2_from_qvn_streamed(q, v, nd, p.n_pop, p.block_id, p.n_block, sink, precision="fixed_i8")
    assert np.array_equal(bs, want.block_sizes)
    assert np.array_equal(f2, want.f2) and np.array_equal(vp, want.vpair)
    n_out = p.n_pop * p.n_pop * p.n_block
    out = (torch.zeros(n_out, dtype=torch.float64, device="cuda"), torch.zeros(n_out, dtype=torch.float64, device="cuda"))
    for src in ((q, v, nd), tuple(torch.as_tensor(x).cuda() for x in (q, v, nd))):
        out[0].zero_()
        out[1].zero_()
        _, _, bs = ctx.f2_from_qvn(*src, p.n_pop, p.block_id, p.n_block, precision="fixed_i8", out=out)
        torch.cuda.synchronize()
        assert np.array_equal(out[0].cpu().numpy(), want.f2) and np.array_equal(out[1].cpu().numpy(), want.vpair)


def test_sink_error_stops_the_call_and_context_recovers(ctx, panel):
    p, sel, po, rec = panel

    class Stop(Exception):
        pass

    def sink(b0, b1, a, v):
        if b0 > 0:
            raise Stop()

    with pytest.raises(Stop):
        ctx.extract_streamed(rec, p.n_ind, sel, po, p.block_id, p.n_block, sink, precision="fixed_i8")
    with pytest.raises(StpError, match="tensor-core"):
        ctx.extract_streamed(rec, p.n_ind, sel, po, p.block_id, p.n_block, lambda *a: None, precision="fp32")
    f2, vp, _, good = _collect(p.n_pop, p.n_block)
    ctx.extract_streamed(rec, p.n_ind, sel, po, p.block_id, p.n_block, good, precision="fixed_i8")
    want = ctx.extract_blocks(rec, p.n_ind, sel, po, p.block_id, p.n_block, precision="fixed_i8")
    assert np.array_equal(f2, want.f2)


def test_extract_f2_disk_tier_writes_the_same_directory(tmp_path):
    p = synth.generate("c1", seed=12, n_snp=20_000, n_pop=9)
    write_eigenstrat(p, tmp_path / "panel")
    pops = sorted(p.pop_labels)
    host = extract_f2(tmp_path / "panel", pops=pops, out=str(tmp_path / "host"), precision="fixed_i8", maxmiss=1.0)
    disk = extract_f2(tmp_path / "panel", pops=pops, out=str(tmp_path / "disk"), precision="fixed_i8", maxmiss=1.0,
                      tier="disk")
    a = (tmp_path / "host" / "f2.bin").read_bytes()
    b = (tmp_path / "disk" / "f2.bin").read_bytes()
    assert a == b
    assert (tmp_path / "host" / "meta.json").read_text() == (tmp_path / "disk" / "meta.json").read_text()
    assert read_f2(host).tensor.n_block == read_f2(disk).tensor.n_block
