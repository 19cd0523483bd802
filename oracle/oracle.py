"""TEST INFRASTRUCTURE ONLY — ctypes access to the CPU checkers built by oracle/Makefile.

``port`` is liboracle.so (the C restatement in f2_oracle.c); ``ref`` is
_ref/libref_oracle.so (the reference's own CpuBackend compiled in place), present only
where the reference sources were available at build time. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libref_oracle.so"

_P = C.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data


class _Lib:
    def __init__(self, path: Path, prefix: str):
        self.path = path
        self.L = C.CDLL(str(path))
        self.prefix = prefix

    def fn(self, name, res, args):
        f = getattr(self.L, self.prefix + name)
        f.restype = res
        f.argtypes = args
        return f


_port = None
_ref = None


def port() -> _Lib:
    global _port
    if _port is None:
        if not PORT_PATH.exists():
            raise ImportError(f"{PORT_PATH} missing: run `make -C oracle`")
        _port = _Lib(PORT_PATH, "or_")
    return _port


def ref_available() -> bool:
    return REF_PATH.exists()


def ref() -> _Lib:
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise ImportError(f"{REF_PATH} missing (the reference sources were not present at build time)")
        _ref = _Lib(REF_PATH, "ref_")
    return _ref


# ---- the C restatement ---------------------------------------------------------------------

def genotype_code(byte: int, k: int) -> int:
    return port().fn("genotype_code", C.c_int, [C.c_uint8, C.c_int])(byte, k)


def detect_ploidy_pa(records: np.ndarray, sel_rows: np.ndarray) -> np.ndarray:
    rec = np.ascontiguousarray(records, np.uint8)
    sel = np.ascontiguousarray(sel_rows, np.int64)
    out = np.zeros(sel.size, np.int32)
    port().fn("detect_ploidy_pa", None, [_P, C.c_size_t, C.c_size_t, _P, C.c_size_t, _P])(
        _ptr(rec), rec.shape[1], rec.shape[0], _ptr(sel), sel.size, _ptr(out))
    return out


def detect_ploidy_canonical(packed: np.ndarray, bpr: int, n_snp: int, n_ind: int) -> np.ndarray:
    pk = np.ascontiguousarray(packed, np.uint8)
    out = np.zeros(n_ind, np.int32)
    port().fn("detect_ploidy_canonical", None, [_P, C.c_size_t, C.c_size_t, C.c_size_t, _P])(
        _ptr(pk), bpr, n_snp, n_ind, _ptr(out))
    return out


def decode_counts_pa(records, sel_rows, pop_offsets, ploidy=None, default_ploidy=2):
    """(ac2, n) int32 flat [P x M] column-major (index i + P*s)."""
    rec = np.ascontiguousarray(records, np.uint8)
    sel = np.ascontiguousarray(sel_rows, np.int64)
    po = np.ascontiguousarray(pop_offsets, np.int64)
    pl = None if ploidy is None else np.ascontiguousarray(ploidy, np.int32)
    P, M = po.size - 1, rec.shape[0]
    ac2 = np.zeros(P * M, np.int32)
    n = np.zeros(P * M, np.int32)
    port().fn("decode_counts_pa", None, [_P, C.c_size_t, C.c_size_t, _P, _P, C.c_int, _P, C.c_int, _P, _P])(
        _ptr(rec), rec.shape[1], M, _ptr(sel), _ptr(po), P, _ptr(pl), default_ploidy, _ptr(ac2), _ptr(n))
    return ac2, n


def counts_to_qvn(ac2: np.ndarray, n: np.ndarray):
    a = np.ascontiguousarray(ac2, np.int32)
    c = np.ascontiguousarray(n, np.int32)
    q, v, nd = np.zeros(a.size), np.zeros(a.size), np.zeros(a.size)
    port().fn("counts_to_qvn", None, [_P, _P, C.c_size_t, _P, _P, _P])(_ptr(a), _ptr(c), a.size, _ptr(q), _ptr(v), _ptr(nd))
    return q, v, nd


def transpose_pa_to_canonical(records, sel_rows) -> tuple[np.ndarray, int]:
    rec = np.ascontiguousarray(records, np.uint8)
    sel = np.ascontiguousarray(sel_rows, np.int64)
    M = rec.shape[0]
    obpr = (M + 3) // 4
    out = np.zeros(sel.size * obpr, np.uint8)
    port().fn("transpose_pa_to_canonical", None, [_P, C.c_size_t, C.c_size_t, _P, C.c_size_t, _P])(
        _ptr(rec), rec.shape[1], M, _ptr(sel), sel.size, _ptr(out))
    return out, obpr


def decode_af_canonical(packed, bpr, n_snp, pop_offsets, sample_ploidy=None, ploidy=2, detect=False, lib=None):
    pk = np.ascontiguousarray(packed, np.uint8)
    po = np.ascontiguousarray(pop_offsets, np.int64)
    P = po.size - 1
    n_ind = pk.size // bpr if bpr else 0
    sp = None if sample_ploidy is None else np.ascontiguousarray(sample_ploidy, np.int32)
    q, v, n = np.zeros(P * n_snp), np.zeros(P * n_snp), np.zeros(P * n_snp)
    if lib == "ref":
        po_sz = np.ascontiguousarray(po, np.uint64)
        rc = ref().fn("decode_af", C.c_int, [_P, C.c_size_t, C.c_size_t, C.c_size_t, _P, C.c_int, _P, C.c_int,
                                             C.c_int, _P, _P, _P])(
            _ptr(pk), bpr, n_snp, n_ind, _ptr(po_sz), P, _ptr(sp), ploidy, 1 if detect else 0, _ptr(q), _ptr(v), _ptr(n))
        assert rc == 0
    else:
        port().fn("decode_af_canonical", None, [_P, C.c_size_t, C.c_size_t, C.c_size_t, _P, C.c_int, _P, C.c_int,
                                                C.c_int, _P, _P, _P])(
            _ptr(pk), bpr, n_snp, n_ind, _ptr(po), P, _ptr(sp), ploidy, 1 if detect else 0, _ptr(q), _ptr(v), _ptr(n))
    return q, v, n


def compute_f2_blocks(Q, V, N, P, block_id, n_block, lib: str = "port"):
    """Per-block f2/vpair [P*P*B] and block_sizes, from flat [P x M] Q/V/N."""
    Q, V, N = (np.ascontiguousarray(x, np.float64) for x in (Q, V, N))
    M = Q.size // P if P > 0 else 0
    bid = np.ascontiguousarray(block_id, np.int32)
    n = max(P, 0) ** 2 * max(n_block, 0)
    f2, vp = np.zeros(n), np.zeros(n)
    bs = np.zeros(max(n_block, 0), np.int32)
    L = ref() if lib == "ref" else port()
    rc = L.fn("compute_f2_blocks", C.c_int, [_P, _P, _P, C.c_int, C.c_long, _P, C.c_int, _P, _P, _P])(
        _ptr(Q), _ptr(V), _ptr(N), P, M, _ptr(bid), n_block, _ptr(f2), _ptr(vp), _ptr(bs))
    if rc != 0:
        raise ValueError("malformed block partition")
    return f2, vp, bs


def compute_f2_blocks_sharded(Q, V, N, P, block_id, n_block, threads: int | None = None, lib: str = "port",
                              blocks: list[int] | None = None):
    """The same result computed as contiguous block shards on `threads` host threads (the
    reference's whole-block fan-out, f2_blocks_multigpu_core.cpp:40-85). `blocks`
    restricts the work to a subset of block ids (others stay zero)."""
    Q, V, N = (np.ascontiguousarray(x, np.float64) for x in (Q, V, N))
    bid = np.ascontiguousarray(block_id, np.int32)
    threads = threads or os.cpu_count() or 1
    edges = np.flatnonzero(np.diff(bid)) + 1
    starts = np.concatenate([[0], edges]).astype(np.int64)
    ends = np.concatenate([edges, [bid.size]]).astype(np.int64)
    ranges = {int(bid[s]): (int(s), int(e)) for s, e in zip(starts, ends)}
    todo = sorted(ranges) if blocks is None else [b for b in blocks if b in ranges]
    slab = P * P
    f2 = np.zeros(slab * n_block)
    vp = np.zeros(slab * n_block)
    bs = np.zeros(n_block, np.int32)
    L = ref() if lib == "ref" else port()
    fn = L.fn("compute_f2_blocks", C.c_int, [_P, _P, _P, C.c_int, C.c_long, _P, C.c_int, _P, _P, _P])

    def one(b):
        s, e = ranges[b]
        m = e - s
        ids = np.zeros(m, np.int32)
        o_f2 = np.zeros(slab)
        o_vp = np.zeros(slab)
        o_bs = np.zeros(1, np.int32)
        off = P * s * 8
        rc = fn(Q.ctypes.data + off, V.ctypes.data + off, N.ctypes.data + off, P, m, _ptr(ids), 1,
                _ptr(o_f2), _ptr(o_vp), _ptr(o_bs))
        assert rc == 0
        f2[slab * b:slab * (b + 1)] = o_f2
        vp[slab * b:slab * (b + 1)] = o_vp
        bs[b] = o_bs[0]

    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(one, todo))
    return f2, vp, bs


def assign_blocks(chrom, genpos, blgsize, physpos=None, bp_window=2.0e6, lib: str = "port"):
    c = np.ascontiguousarray(chrom, np.int32)
    g = np.ascontiguousarray(genpos, np.float64)
    p = None if physpos is None else np.ascontiguousarray(physpos, np.float64)
    out = np.zeros(max(c.size, 1), np.int32)
    L = ref() if lib == "ref" else port()
    nb = L.fn("assign_blocks", C.c_int, [_P, _P, C.c_long, C.c_double, _P, C.c_double, _P])(
        _ptr(c), _ptr(g), c.size, blgsize, _ptr(p), bp_window, _ptr(out))
    return out[: c.size] if nb > 0 else np.zeros(0, np.int32), nb


def block_jackknife(x, block_sizes, m, nb, lib: str = "port"):
    x = np.ascontiguousarray(x, np.float64)
    bs = np.ascontiguousarray(block_sizes, np.int32)
    est, var = np.zeros(m), np.zeros(m)
    if lib == "ref":
        rc = ref().fn("block_jackknife", C.c_int, [_P, _P, C.c_long, C.c_int, _P, _P])(
            _ptr(x), _ptr(bs), m, nb, _ptr(est), _ptr(var))
        assert rc == 0
    else:
        port().fn("block_jackknife", None, [_P, _P, C.c_long, C.c_int, _P, _P])(
            _ptr(x), _ptr(bs), m, nb, _ptr(est), _ptr(var))
    return est, var


def f2_from_panel(records, sel_rows, pop_offsets, block_id, n_block, ploidy=None, lib: str = "port",
                  threads: int | None = None):
    """Full CPU extraction on SNP-major records: decode (counts) -> q/v/n -> per-block f2."""
    ac2, n = decode_counts_pa(records, sel_rows, pop_offsets, ploidy)
    q, v, nd = counts_to_qvn(ac2, n)
    P = len(pop_offsets) - 1
    if threads is not None and threads > 1:
        return compute_f2_blocks_sharded(q, v, nd, P, block_id, n_block, threads, lib)
    return compute_f2_blocks(q, v, nd, P, block_id, n_block, lib)


def survivor_blocks(vpair, P, nb):
    """cpu_backend.cpp:124-151: keep flags per block."""
    vp = np.ascontiguousarray(vpair, np.float64)
    keep = np.zeros(max(nb, 1), np.int32)
    port().fn("survivor_blocks", C.c_int, [_P, C.c_int, C.c_int, _P])(_ptr(vp), P, nb, _ptr(keep))
    return keep[:nb].astype(bool)


FSTAT_KINDS = {"f4": 0, "f3": 1, "f4_lr": 2}


def fstats(f2, vpair, block_sizes, P, nb, kind, idx, n_stat, lib: str = "port", with_blocks: bool = False):
    """f4 quartets / f3 triples / f4 left-right statistics with their block jackknife over
    the surviving blocks (see or_fstats). Returns (est, var, n_survivors[, x_blocks])."""
    k = FSTAT_KINDS[kind] if isinstance(kind, str) else int(kind)
    f2 = np.ascontiguousarray(f2, np.float64)
    vp = np.ascontiguousarray(vpair, np.float64)
    bs = np.ascontiguousarray(block_sizes, np.int32)
    ix = np.ascontiguousarray(idx, np.int32)
    if k == 2:
        m = max(n_stat - 1, 0) * max(ix.size - n_stat - 1, 0)
    else:
        m = n_stat
    est, var = np.zeros(max(m, 1)), np.zeros(max(m, 1))
    if lib == "ref":
        ns = ref().fn("fstats", C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_long, C.c_long, _P, _P])(
            _ptr(f2), _ptr(vp), _ptr(bs), P, nb, k, _ptr(ix), ix.size, n_stat, _ptr(est), _ptr(var))
        if ns < 0:
            raise ValueError("reference f-statistics failed")
        return est[:m], var[:m], ns
    xb = np.zeros(max(m, 1) * max(nb, 1))
    ns = port().fn("fstats", C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_long, C.c_long, _P, _P, _P])(
        _ptr(f2), _ptr(vp), _ptr(bs), P, nb, k, _ptr(ix), ix.size, n_stat, _ptr(est), _ptr(var), _ptr(xb))
    out = (est[:m], var[:m], ns)
    return out + (xb[:m * ns].reshape(ns, m),) if with_blocks else out


def keep_mask(Q, N, P, ref_alleles, alt_alleles, chrom, maf_min=0.0, maxmiss=1.0, autosomes_only=False, drop_monomorphic=False,
              transversions_only=False, strand_mode=0, total_indiv=None, lib: str = "port"):
    """extract-f2's per-SNP keep mask from Q / N [P x M] (flat, i + P*s) and the .snp alleles /
    chromosomes. Returns (keep uint8 [M], summary float64 [4, M]: ref AF, minor AF, missing
    fraction, allele count). total_indiv defaults to the called-allele capacity / 2 of the
    selection (pass the selection's individual count)."""
    Qa = np.ascontiguousarray(Q, np.float64)
    Na = np.ascontiguousarray(N, np.float64)
    M = Qa.size // P if P > 0 else 0
    def codes(x):  # allele characters as uint8 codes (from codes or from characters)
        x = np.asarray(x)
        if x.dtype in (np.uint8, np.int8):
            return np.ascontiguousarray(x.view(np.uint8))
        return np.ascontiguousarray(np.asarray(x, dtype="S1").view(np.uint8))

    r, a = codes(ref_alleles), codes(alt_alleles)
    c = np.ascontiguousarray(chrom, np.int32)
    keep = np.zeros(max(M, 1), np.uint8)
    summ = np.zeros(4 * max(M, 1))
    args = [_P, _P, C.c_int, C.c_long, _P, _P, _P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
            C.c_double, _P, _P]
    vals = (_ptr(Qa), _ptr(Na), P, M, _ptr(r), _ptr(a), _ptr(c), float(maf_min), float(maxmiss), int(autosomes_only),
            int(drop_monomorphic), int(transversions_only), int(strand_mode), float(total_indiv), _ptr(keep),
            _ptr(summ))
    if lib == "ref":
        rc = ref().fn("keep_mask", C.c_int, args)(*vals)
        assert rc == 0
    else:
        port().fn("keep_mask", None, args)(*vals)
    return keep[:M], summ[:4 * M].reshape(4, M)
