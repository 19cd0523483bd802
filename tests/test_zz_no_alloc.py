"""The allocation-free count decode (stp_decode_counts_noalloc).

Some callers cannot allocate device memory at call time: a process whose memory pool or
caching allocator already holds the free HBM (a cudaMalloc there fails or makes the pool
give memory back and synchronise), or a caller on a latency-critical stream (cudaFree
synchronises the whole device). This entry point serves them from one static device array.

Checked here, through the C ABI on the GPU, on two calls in a row: the counts equal the
oracle's and the allocating stp_decode_counts bit for bit (counts are integers, so the
tolerance is equality), and the device's free memory is the same before and after a call.

Collected last on purpose (file name): it runs after every other GPU test has used the
library, and also passes on its own in a fresh process.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from steppecu_b200 import StpError, synth

pytestmark = pytest.mark.gpu


def _device_records(rec: np.ndarray):
    import torch

    pitch = (rec.shape[1] + 15) // 16 * 16
    h = np.zeros((rec.shape[0], pitch), dtype=np.uint8)
    h[:, :rec.shape[1]] = rec
    d = torch.as_tensor(h).cuda()
    torch.cuda.synchronize()
    return d


@pytest.mark.parametrize("ploidy", ["auto", "diploid", "given"])
def test_noalloc_counts_equal_oracle_and_decode_counts_twice(ctx, ploidy):
    import torch

    p = synth.generate("c4", seed=23, n_snp=20_000, n_pop=37)
    sel, po = p.selection()
    rec = p.records_numpy()
    given = np.where(np.arange(sel.size) % 3 == 0, 2, 1).astype(np.int32) if ploidy == "given" else None
    mode = "auto" if ploidy == "given" else ploidy
    P, M = len(po) - 1, p.n_snp
    if given is not None:
        pl = given
    elif mode == "diploid":
        pl = np.full(sel.size, 2, np.int32)
    else:
        pl = oracle.detect_ploidy_pa(rec, sel)
    o_ac2, o_n = oracle.decode_counts_pa(rec, sel, po, pl)
    o_ac2, o_n = o_ac2.reshape(-1, P).T, o_n.reshape(-1, P).T
    want_ac2, want_n = ctx.decode_counts(rec, p.n_ind, sel, po, sample_ploidy=given, ploidy=mode)
    assert np.array_equal(want_ac2, o_ac2) and np.array_equal(want_n, o_n)

    d_rec = _device_records(rec)
    stream = torch.cuda.Stream()
    ac2 = torch.empty(M * P, dtype=torch.int32, device="cuda")
    n = torch.empty(M * P, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free = []
    for _ in range(2):  # two calls in a row through the same static scratch
        with torch.cuda.stream(stream):
            ac2.fill_(-7)
            n.fill_(-7)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        ctx.decode_counts_noalloc(d_rec, p.n_ind, sel, po, ac2, n, sample_ploidy=given, ploidy=mode,
                                  stream=stream)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        assert np.array_equal(ac2.cpu().numpy().reshape(M, P).T, o_ac2)
        assert np.array_equal(n.cpu().numpy().reshape(M, P).T, o_n)
    # The first call may map the library's static array on this device; from then on a call
    # changes nothing in the device's free memory.
    assert free[2] == free[3], free


def test_noalloc_default_stream_follows_torch_current_stream(ctx):
    import torch

    p = synth.generate("c1", seed=5, n_snp=3000, n_pop=6)
    sel, po = p.selection()
    rec = p.records_numpy()
    want_ac2, want_n = ctx.decode_counts(rec, p.n_ind, sel, po)
    P, M = len(po) - 1, p.n_snp
    d_rec = _device_records(rec)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        ac2 = torch.full((M * P,), -7, dtype=torch.int32, device="cuda")
        n = torch.full((M * P,), -7, dtype=torch.int32, device="cuda")
        ctx.decode_counts_noalloc(d_rec, p.n_ind, sel, po, ac2, n)  # runs after the fills on s
    torch.cuda.synchronize()
    assert np.array_equal(ac2.cpu().numpy().reshape(M, P).T, want_ac2)
    assert np.array_equal(n.cpu().numpy().reshape(M, P).T, want_n)


def test_noalloc_rejects_wrong_output_buffers(ctx):
    import torch

    p = synth.generate("c1", seed=3, n_snp=500, n_pop=3)
    sel, po = p.selection()
    d_rec = _device_records(p.records_numpy())
    good = torch.zeros(3 * 500, dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError, match="int32"):
        ctx.decode_counts_noalloc(d_rec, p.n_ind, sel, po, good.to(torch.int64), good)
    with pytest.raises(ValueError, match="elements"):
        ctx.decode_counts_noalloc(d_rec, p.n_ind, sel, po, good[:100], good)
    with pytest.raises(ValueError, match="uint8"):
        ctx.decode_counts_noalloc(d_rec.to(torch.int32), p.n_ind, sel, po, good, good)


def test_noalloc_rejects_requests_over_the_scratch(ctx):
    import torch

    # 4,000 selected samples x 200,000 SNPs needs ~200 MB of canonical genotypes: refused
    # before any device work (the records tensor is never read).
    n_ind, M = 4000, 200_000
    d_rec = torch.zeros((M, 1008), dtype=torch.uint8, device="cuda")
    sel = np.arange(n_ind, dtype=np.int64)
    po = np.array([0, 2000, 4000], dtype=np.int64)
    out = torch.zeros(2 * M, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(StpError, match="scratch"):
        ctx.decode_counts_noalloc(d_rec, n_ind, sel, po, out, out)


def test_noalloc_rejects_unaligned_pitch(ctx):
    import torch

    p = synth.generate("c1", seed=3, n_snp=500, n_pop=3)
    sel, po = p.selection()
    rec = p.records_numpy()
    d = torch.as_tensor(rec).cuda()
    if rec.shape[1] % 16 == 0:
        d = torch.zeros((rec.shape[0], rec.shape[1] + 1), dtype=torch.uint8, device="cuda")
    out = torch.zeros(3 * 500, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(StpError, match="16-byte"):
        ctx.decode_counts_noalloc(d, p.n_ind, sel, po, out, out)
