"""The allocation-free count decode (stp_decode_counts_noalloc) against stp_decode_counts.

Collected last on purpose (file name): it runs after every other GPU test has used the
library, and also passes on its own. Counts are integers, so "within tolerance" is equality.
"""
from __future__ import annotations

import numpy as np
import pytest

from steppecu_b200 import StpError, synth

pytestmark = pytest.mark.gpu


def _device_records(rec: np.ndarray):
    import torch

    pitch = (rec.shape[1] + 15) // 16 * 16
    d = torch.zeros((rec.shape[0], pitch), dtype=torch.uint8, device="cuda")
    d[:, :rec.shape[1]] = torch.as_tensor(rec).cuda()
    return d


@pytest.mark.parametrize("ploidy", ["auto", "diploid", "given"])
def test_noalloc_counts_equal_decode_counts_twice(ctx, ploidy):
    import torch

    p = synth.generate("c4", seed=23, n_snp=20_000, n_pop=37)
    sel, po = p.selection()
    rec = p.records_numpy()
    given = np.where(np.arange(sel.size) % 3 == 0, 2, 1).astype(np.int32) if ploidy == "given" else None
    mode = "auto" if ploidy == "given" else ploidy
    want_ac2, want_n = ctx.decode_counts(rec, p.n_ind, sel, po, sample_ploidy=given, ploidy=mode)
    d_rec = _device_records(rec)
    P, M = len(po) - 1, p.n_snp
    for _ in range(2):  # two calls in a row through the same static scratch
        ac2 = torch.full((M * P,), -7, dtype=torch.int32, device="cuda")
        n = torch.full((M * P,), -7, dtype=torch.int32, device="cuda")
        ctx.decode_counts_noalloc(d_rec, p.n_ind, sel, po, ac2, n, sample_ploidy=given, ploidy=mode)
        torch.cuda.synchronize()
        assert np.array_equal(ac2.cpu().numpy().reshape(M, P).T, want_ac2)
        assert np.array_equal(n.cpu().numpy().reshape(M, P).T, want_n)


def test_noalloc_rejects_requests_over_the_scratch(ctx):
    import torch

    # 4,000 selected samples x 200,000 SNPs needs ~200 MB of canonical genotypes: refused
    # before any device work (the records tensor is never read).
    n_ind, M = 4000, 200_000
    d_rec = torch.zeros((M, 1008), dtype=torch.uint8, device="cuda")
    sel = np.arange(n_ind, dtype=np.int64)
    po = np.array([0, 2000, 4000], dtype=np.int64)
    out = torch.zeros(2 * M, dtype=torch.int32, device="cuda")
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
    with pytest.raises(StpError, match="16-byte"):
        ctx.decode_counts_noalloc(d, p.n_ind, sel, po, out, out)
