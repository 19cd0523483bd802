"""The fixed-point arithmetic of the STP_PREC_FIXED_I8 contraction, restated in numpy and
checked exhaustively against exact f2 terms (CPU only; the GPU parity tests check the
kernels themselves).

Per population and SNP the decode stores X = round((q - 1/2) S) and -A with A =
round((x^2 - h) S^2 / 2^31), S = 127 * 2^25, as four balanced int8 digits each, and M = 64
[n > 0]; the contraction sums, exactly in int32, the digit products of X of weight >= 256^3
and the products of A's digits with M; f2's per-SNP term is -2 / S^2 times that bracket.
Over every pair of frequencies a population of up to 20 diploid samples can have (n up to
40 called alleles), the per-SNP error of that term must stay below 1e-9: the absolute
floor of the tolerance holds even for one-SNP blocks, by construction.
"""
from __future__ import annotations

import numpy as np

S = 127.0 * 2.0**25
SA = 16129.0 * 2.0**19  # S^2 / 2^31


def _digits(v: np.ndarray) -> list[np.ndarray]:
    """Balanced base-256 digits, least significant first: the bytes of (v + 0x80808080),
    each minus 128 (the decode's (v + 0x80808080) ^ 0x80808080 read as int8)."""
    y = (v.astype(np.int64) + 0x80808080) & 0xFFFFFFFF
    return [((y >> (8 * k)) & 0xFF) - 128 for k in range(4)]


def _all_frequencies(n_max: int = 40):
    q, h = [], []
    for n in range(1, n_max + 1):
        for a2 in range(0, 2 * n + 1):
            qq = a2 * 0.5 / n
            q.append(qq)
            h.append(qq * (1.0 - qq) / max(n - 1, 1))
    return np.array(q), np.array(h)


def test_digits_reconstruct_and_stay_in_range():
    q, h = _all_frequencies()
    x = q - 0.5
    X = np.rint(x * S).astype(np.int64)
    A = np.rint((x * x - h) * SA).astype(np.int64)
    for v in (X, -A):
        d = _digits(v)
        assert np.array_equal(sum(d[k] * 256**k for k in range(4)), v)
        assert all(((dk >= -128) & (dk <= 127)).all() for dk in d)
    # Four digit products and two digit-times-64 products per SNP at the lowest weight keep
    # the int32 accumulators exact over a 16,384-SNP segment.
    assert 16_384 * (4 * 128 * 128 + 2 * 128 * 64) < 2**31


def test_per_snp_term_error_below_floor():
    q, h = _all_frequencies()
    x = q - 0.5
    X = np.rint(x * S).astype(np.int64)
    NA = np.rint(-(x * x - h) * SA).astype(np.int64)
    dx, de = _digits(X), _digits(NA)
    i, j = np.meshgrid(np.arange(q.size), np.arange(q.size), indexing="ij")
    i, j = i.ravel(), j.ravel()
    bracket = np.zeros(i.size)
    for a in range(4):
        for b in range(4):
            if a + b >= 3:
                bracket += (dx[a][i] * dx[b][j]).astype(np.float64) * 256.0 ** (a + b)
    for k in range(4):
        # E_k(i) M(j) + M(i) E_k(j), M = 64 (both called), at weight 256^(3+k)
        bracket += 64.0 * (de[k][i] + de[k][j]).astype(np.float64) * 256.0 ** (3 + k)
    term = -2.0 * bracket / S**2
    exact = (q[i] - q[j]) ** 2 - h[i] - h[j]
    err = np.abs(term - exact)
    assert err.max() < 1e-9, err.max()
