"""Python surface of the B200 f2 extraction, mirroring the reference's bindings.

``extract_f2`` / ``read_f2`` / ``F2Blocks`` follow ``steppe.extract_f2``, ``steppe.read_f2``
and the ``F2Handle`` opaque type (bindings/steppe/__init__.py:493-560,
bindings/bind_f2handle.cpp:26-47, bindings/bind_fstats.cpp:130-224 in the reference).
``Context`` exposes the C-ABI entry points that stand in for the ComputeBackend
f2/decode virtuals. Every computation runs in libstpf2.so on the GPU; without a CUDA
device the calls raise, as the reference does.
"""
from __future__ import annotations

import ctypes as C
import weakref
from pathlib import Path

import numpy as np

from . import _lib as L
from .blocks import assign_blocks
from .eigenstrat import read_geno, read_ind, read_snp, select_pops
from .f2dir import F2DirWriter, F2Tensor, read_f2_dir, write_f2_dir

PRECISIONS = {
    "fp32": L.PREC_FP32_SIMT, "fp32_simt": L.PREC_FP32_SIMT, "simt": L.PREC_FP32_SIMT,
    "bf16x3": L.PREC_SPLIT_BF16, "split_bf16": L.PREC_SPLIT_BF16, "bf16": L.PREC_SPLIT_BF16,
    "f16x3": L.PREC_SPLIT_F16, "split_f16": L.PREC_SPLIT_F16, "fp16": L.PREC_SPLIT_F16,
    "split_f16_fine": L.PREC_SPLIT_F16_FINE, "f16x3_fine": L.PREC_SPLIT_F16_FINE,
    "fixed_i8": L.PREC_FIXED_I8, "i8x4": L.PREC_FIXED_I8,
}
PRECISION_TAGS = {L.PREC_FP32_SIMT: "fp32_simt", L.PREC_SPLIT_BF16: "split_bf16", L.PREC_SPLIT_F16: "split_f16",
                  L.PREC_SPLIT_F16_FINE: "split_f16_fine", L.PREC_FIXED_I8: "fixed_i8"}
DEFAULT_PRECISION = "fixed_i8"

PLOIDY = {"auto": L.PLOIDY_AUTO, "1": L.PLOIDY_PSEUDO, "pseudo": L.PLOIDY_PSEUDO,
          "pseudo_haploid": L.PLOIDY_PSEUDO, "2": L.PLOIDY_DIPLOID, "diploid": L.PLOIDY_DIPLOID}


STRAND = {"drop": L.STRAND_DROP, "keep": L.STRAND_KEEP, "flip": L.STRAND_FLIP}


def snp_filter(maf_min: float = 0.0, maxmiss: float = 1.0, autosomes_only: bool = False,
               drop_monomorphic: bool = False, transversions_only: bool = False,
               strand_mode: str = "drop") -> L.SnpFilter:
    """The stp_snp_filter of extract-f2's per-SNP filters (FilterConfig)."""
    if strand_mode not in STRAND:
        raise ValueError("strand_mode must be one of 'drop', 'keep', 'flip'")
    return L.SnpFilter(float(maf_min), float(maxmiss), int(bool(autosomes_only)), int(bool(drop_monomorphic)),
                       int(bool(transversions_only)), STRAND[strand_mode])


def parse_precision(precision) -> int:
    if precision is None:
        precision = DEFAULT_PRECISION
    if isinstance(precision, int):
        return precision
    try:
        return PRECISIONS[str(precision)]
    except KeyError:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)} (got {precision!r})") from None


def _alleles(x) -> np.ndarray:
    """Per-SNP allele characters as uint8 codes (from a uint8 code array or characters)."""
    a = np.asarray(x)
    if a.dtype in (np.uint8, np.int8):
        return np.ascontiguousarray(a.view(np.uint8))
    return np.ascontiguousarray(np.asarray(a, dtype="S1").view(np.uint8))


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _data_ptr(x) -> int:
    return int(x.data_ptr()) if hasattr(x, "data_ptr") else int(x.ctypes.data)


class Context:
    """One libstpf2 context (make_cuda_backend(device)): a device and a CUDA stream."""

    def __init__(self, device: int = 0):
        st = C.c_int(0)
        self._h = L.lib().stp_create(device, C.byref(st))
        if not self._h:
            raise L.StpError(st.value, L.lib().stp_last_error().decode())
        self.device = device
        self._plans = weakref.WeakSet()  # live plans, closed before the context
        from steppecu_b200.autotune import load_mask

        mask = load_mask()  # the measured tile-class table, when one is committed
        if mask is not None:
            self.set_tile_classes(mask)

    def close(self):
        """Destroys the context, after every plan still open on it (a plan uses the
        context's stream and workspaces, so the C API frees plans first)."""
        if getattr(self, "_h", None):
            for plan in list(getattr(self, "_plans", ())):
                plan.close()
            L.lib().stp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def launches(self) -> int:
        return int(L.lib().stp_launch_count(self._h))

    def set_wait_bounds(self, timeout_ns: int = 0, withhold_stage: int = -1) -> None:
        """stp_set_wait_bounds: the device-side wait bound of the fixed-point contraction
        (0 = default) and its test hook (withhold_stage >= 0 starves the MMA issuer)."""
        L.check(L.lib().stp_set_wait_bounds(self._h, int(timeout_ns), int(withhold_stage)))

    def set_tile_classes(self, partial_feed_mask: int) -> None:
        """stp_set_tile_classes: bit k makes a tile side of 8k+1 .. 8k+8 valid populations stage
        only its valid rows (steppecu_b200/autotune.py measures the choice)."""
        L.check(L.lib().stp_set_tile_classes(self._h, int(partial_feed_mask) & 0xFFFF))

    # -- genotype views ---------------------------------------------------------------
    @staticmethod
    def geno_view(records, n_ind: int, bytes_per_record: int | None = None) -> L.GenoView:
        """records: numpy uint8 [n_snp, pitch] (host) or a torch CUDA uint8 tensor."""
        n_snp = int(records.shape[0])
        pitch = int(records.shape[1]) if records.ndim == 2 else 0
        bpr = bytes_per_record or max(48, (n_ind + 3) // 4)
        if not _is_torch_cuda(records):
            records = np.ascontiguousarray(records)
        v = L.GenoView(_data_ptr(records), bpr, pitch, n_snp, n_ind, 1 if _is_torch_cuda(records) else 0)
        v._keep = records
        return v

    # -- decode ---------------------------------------------------------------------------
    def detect_ploidy(self, records, n_ind: int, sel_rows) -> np.ndarray:
        v = self.geno_view(records, n_ind)
        sel = _i64(sel_rows)
        out = np.zeros(sel.size, np.int32)
        L.check(L.lib().stp_detect_ploidy(self._h, C.byref(v), L.ptr(sel), sel.size, L.ptr(out)))
        return out

    def detect_ploidy_tile(self, packed, bytes_per_record: int, n_snp: int) -> np.ndarray:
        """detect_sample_ploidy_device on the canonical individual-major tile: one record of
        bytes_per_record bytes per individual, SNP codes MSB-first."""
        pk = np.ascontiguousarray(packed, dtype=np.uint8)
        n_ind = pk.size // bytes_per_record if bytes_per_record else 0
        out = np.zeros(n_ind, np.int32)
        L.check(L.lib().stp_detect_ploidy_tile(self._h, L.ptr(pk), bytes_per_record, n_snp, n_ind, 0, L.ptr(out)))
        return out

    def decode_counts(self, records, n_ind: int, sel_rows, pop_offsets, sample_ploidy=None,
                      ploidy: str | int = "auto") -> tuple[np.ndarray, np.ndarray]:
        """(ac2, n) int32 [P, M] C-order views of the column-major [P x M] counts."""
        v = self.geno_view(records, n_ind)
        sel, po = _i64(sel_rows), _i64(pop_offsets)
        P = po.size - 1
        M = v.n_snp
        ac2 = np.zeros(P * M, np.int32)
        n = np.zeros(P * M, np.int32)
        sp = None if sample_ploidy is None else _i32(sample_ploidy)
        mode = PLOIDY[str(ploidy)] if not isinstance(ploidy, int) else ploidy
        L.check(L.lib().stp_decode_counts(self._h, C.byref(v), L.ptr(sel), L.ptr(po), P, L.ptr(sp), mode,
                                          L.ptr(ac2), L.ptr(n)))
        return ac2.reshape(M, P).T, n.reshape(M, P).T

    def decode_counts_noalloc(self, d_records, n_ind: int, sel_rows, pop_offsets, d_ac2, d_n,
                              sample_ploidy=None, ploidy: str | int = "auto", stream=None) -> None:
        """stp_decode_counts_noalloc: device records (torch CUDA uint8 [n_snp, pitch], pitch a
        multiple of 16) -> the caller's device int32 buffers d_ac2 / d_n (n_pop * n_snp each,
        column-major like decode_counts). Allocates nothing on the device."""
        import torch

        if not (_is_torch_cuda(d_records) and _is_torch_cuda(d_ac2) and _is_torch_cuda(d_n)):
            raise TypeError("decode_counts_noalloc takes torch CUDA tensors")
        sel, po = _i64(sel_rows), _i64(pop_offsets)
        P = po.size - 1
        if d_records.dtype != torch.uint8 or not d_records.is_contiguous() or d_records.dim() != 2:
            raise ValueError("d_records must be a contiguous uint8 CUDA tensor [n_snp, pitch]")
        need = max(P, 0) * d_records.shape[0]
        for name, t in (("d_ac2", d_ac2), ("d_n", d_n)):
            if t.dtype != torch.int32 or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous int32 CUDA tensor")
            if t.numel() < need:
                raise ValueError(f"{name} holds {t.numel()} elements; n_pop * n_snp = {need} are written")
            if t.device.index != self.device or d_records.device.index != self.device:
                raise ValueError(f"{name} and d_records must be on this context's device cuda:{self.device}")
        v = self.geno_view(d_records, n_ind)
        sp = None if sample_ploidy is None else _i32(sample_ploidy)
        mode = PLOIDY[str(ploidy)] if not isinstance(ploidy, int) else ploidy
        # Work is ordered after what torch queued on the current stream (the records upload,
        # the output tensors' fills) unless the caller names a stream.
        if stream is None:
            stream = torch.cuda.current_stream(self.device)
        st = C.c_void_p(stream.cuda_stream)
        L.check(L.lib().stp_decode_counts_noalloc(self._h, C.byref(v), L.ptr(sel), L.ptr(po), po.size - 1,
                                                  L.ptr(sp), mode, C.c_void_p(d_ac2.data_ptr()),
                                                  C.c_void_p(d_n.data_ptr()), st))

    def decode_af(self, packed, bytes_per_record: int, n_snp: int, pop_offsets, sample_ploidy=None,
                  ploidy: int = 2, detect: bool = False):
        """ComputeBackend::decode_af on the canonical individual-major tile. Returns flat
        column-major [P x M] q, v, n (FP64), index i + P*s."""
        po = _i64(pop_offsets)
        P = po.size - 1
        pk = np.ascontiguousarray(packed, dtype=np.uint8)
        n_ind = pk.size // bytes_per_record if bytes_per_record else 0
        q = np.zeros(P * n_snp)
        v = np.zeros(P * n_snp)
        n = np.zeros(P * n_snp)
        sp = None if sample_ploidy is None else _i32(sample_ploidy)
        L.check(L.lib().stp_decode_af(self._h, L.ptr(pk), bytes_per_record, n_snp, n_ind, L.ptr(po), P,
                                      L.ptr(sp), ploidy, 1 if detect else 0, 0, L.ptr(q), L.ptr(v), L.ptr(n)))
        return q, v, n

    # -- f2 ---------------------------------------------------------------------------------
    def f2_from_qvn(self, Q, V, N, P: int, block_id, n_block: int, precision=None, out=None) -> F2Tensor:
        """ComputeBackend::compute_f2_blocks(MatView Q, V, N, ...): flat [P x M] inputs. With
        out = (f2, vpair) torch CUDA tensors the result stays on the device
        (compute_f2_blocks_device, stp_f2_from_qvn_device); Q / V / N may then be torch CUDA
        tensors too. Returns the F2Tensor, or (f2, vpair, block_sizes) for device output."""
        bid = _i32(block_id)
        if out is not None:
            on_dev = _is_torch_cuda(Q)
            if not on_dev:
                Q, V, N = (np.ascontiguousarray(x, dtype=np.float64) for x in (Q, V, N))
            M = (Q.numel() if on_dev else Q.size) // P if P > 0 else 0
            bs = np.zeros(max(n_block, 0), np.int32)
            L.check(L.lib().stp_f2_from_qvn_device(self._h, _data_ptr(Q), _data_ptr(V), _data_ptr(N), P, M, L.ptr(bid),
                                                   n_block, parse_precision(precision), 1 if on_dev else 0,
                                                   _data_ptr(out[0]), _data_ptr(out[1]), L.ptr(bs)))
            return out[0], out[1], bs
        Q, V, N = (np.ascontiguousarray(x, dtype=np.float64) for x in (Q, V, N))
        M = Q.size // P if P > 0 else 0
        n = P * P * n_block
        f2 = np.zeros(n)
        vp = np.zeros(n)
        bs = np.zeros(max(n_block, 0), np.int32)
        L.check(L.lib().stp_f2_from_qvn(self._h, L.ptr(Q), L.ptr(V), L.ptr(N), P, M, L.ptr(bid), n_block,
                                        parse_precision(precision), L.ptr(f2), L.ptr(vp), L.ptr(bs)))
        return F2Tensor(f2, vp, bs, P, n_block)

    def _request(self, records, n_ind, sel_rows, pop_offsets, block_id, n_block, precision,
                 sample_ploidy=None, ploidy="auto", kept_rows=None):
        v = self.geno_view(records, n_ind)
        sel, po, bid = _i64(sel_rows), _i64(pop_offsets), _i32(block_id)
        sp = None if sample_ploidy is None else _i32(sample_ploidy)
        kr = None if kept_rows is None else _i64(kept_rows)
        mode = PLOIDY[str(ploidy)] if not isinstance(ploidy, int) else ploidy
        r = L.F2Request(v, L.ptr(sel), L.ptr(po), po.size - 1, L.ptr(sp), mode, L.ptr(bid), n_block,
                        parse_precision(precision), L.ptr(kr), 0 if kr is None else kr.size)
        r._keep = (v, sel, po, bid, sp, kr)
        return r

    def snp_keep_mask(self, records, n_ind: int, sel_rows, pop_offsets, ref, alt, chrom, *, maf_min: float = 0.0,
                      maxmiss: float = 1.0, autosomes_only: bool = False, drop_monomorphic: bool = False,
                      transversions_only: bool = False, strand_mode: str = "drop", sample_ploidy=None,
                      ploidy="auto", summary: bool = False):
        """stp_snp_keep_mask: extract-f2's per-SNP keep mask on the device (bool [n_snp]), and
        with summary=True also the pooled summary [4, n_snp] (ref AF, minor AF, missing
        fraction, allele count). ref / alt: per-SNP allele characters; chrom: int codes."""
        v = self.geno_view(records, n_ind)
        sel, po = _i64(sel_rows), _i64(pop_offsets)
        sp = None if sample_ploidy is None else _i32(sample_ploidy)
        mode = PLOIDY[str(ploidy)] if not isinstance(ploidy, int) else ploidy
        M = v.n_snp
        r = np.ascontiguousarray(_alleles(ref)[:M])
        a = np.ascontiguousarray(_alleles(alt)[:M])
        c = _i32(np.asarray(chrom)[:M])
        if r.size < M or a.size < M or c.size < M:
            raise ValueError("ref / alt / chrom need one entry per SNP")
        f = snp_filter(maf_min, maxmiss, autosomes_only, drop_monomorphic, transversions_only, strand_mode)
        keep = np.zeros(max(M, 1), np.uint8)
        summ = np.zeros(4 * M) if summary else None
        n_kept = C.c_int64(0)
        L.check(L.lib().stp_snp_keep_mask(self._h, C.byref(v), L.ptr(sel), L.ptr(po), po.size - 1, L.ptr(sp), mode,
                                          L.ptr(r), L.ptr(a), L.ptr(c), C.byref(f), L.ptr(keep), C.byref(n_kept),
                                          L.ptr(summ)))
        k = keep[:M].astype(bool)
        return (k, summ.reshape(4, M)) if summary else k

    def canonical_to_records(self, packed, bytes_per_record: int, n_snp: int, n_ind: int, d_records) -> None:
        """stp_canonical_to_records: a host canonical individual-major tile into SNP-major
        records in the torch CUDA uint8 tensor d_records [n_snp, pitch]."""
        pk = np.ascontiguousarray(packed, dtype=np.uint8)
        L.check(L.lib().stp_canonical_to_records(self._h, L.ptr(pk), bytes_per_record, n_snp, n_ind, 0,
                                                 _data_ptr(d_records), int(d_records.shape[1])))

    def decode_af_compact_filter(self, packed, bytes_per_record: int, n_snp: int, pop_offsets, ref, alt, chrom,
                                 filt: dict | None = None, sample_ploidy=None, ploidy: int = 2,
                                 total_indiv: float | None = None):
        """stp_decode_af_compact_filter on a canonical individual-major tile: (keep [n_snp],
        q, v, n flat [P x n_kept])."""
        po = _i64(pop_offsets)
        P = po.size - 1
        pk = np.ascontiguousarray(packed, dtype=np.uint8)
        n_ind = pk.size // bytes_per_record if bytes_per_record else 0
        r = _alleles(ref)
        a = _alleles(alt)
        c = _i32(chrom)
        f = snp_filter(**(filt or {}))
        sp = None if sample_ploidy is None else _i32(sample_ploidy)
        tot = float(po[-1] if total_indiv is None else total_indiv)
        keep = np.zeros(max(n_snp, 1), np.uint8)
        nk = C.c_int64(0)
        lib = L.lib()
        args = (self._h, L.ptr(pk), bytes_per_record, n_snp, n_ind, L.ptr(po), P, L.ptr(sp), ploidy, 0, L.ptr(r),
                L.ptr(a), L.ptr(c), C.byref(f), tot, L.ptr(keep), C.byref(nk))
        L.check(lib.stp_decode_af_compact_filter(*args, None, None, None, 0))
        q, v, n = (np.zeros(max(P * nk.value, 1)) for _ in range(3))
        L.check(lib.stp_decode_af_compact_filter(*args, L.ptr(q), L.ptr(v), L.ptr(n), 0))
        m = P * nk.value
        return keep[:n_snp].astype(bool), q[:m], v[:m], n[:m]

    def extract_blocks(self, records, n_ind: int, sel_rows, pop_offsets, block_id, n_block: int,
                       precision=None, sample_ploidy=None, ploidy="auto", out=None,
                       return_ploidy: bool = False, kept_rows=None):
        """The extract-f2 hot path on one request. records: host numpy [M, bpr] or a torch
        CUDA tensor. out: optional (f2, vpair) buffers (numpy host or torch CUDA). kept_rows:
        optional strictly increasing record rows of the SNPs to extract (block_id then has
        one entry per kept row); the decode reads them in place."""
        r = self._request(records, n_ind, sel_rows, pop_offsets, block_id, n_block, precision,
                          sample_ploidy, ploidy, kept_rows)
        P = r.n_pop
        n = P * P * n_block
        if out is None:
            f2, vp = np.zeros(n), np.zeros(n)
        else:
            f2, vp = out
        on_dev = _is_torch_cuda(f2)
        bs = np.zeros(max(n_block, 0), np.int32)
        ploidy_out = np.zeros(int(r._keep[1].size), np.int32) if return_ploidy else None
        o = L.F2Output(_data_ptr(f2), _data_ptr(vp), L.ptr(bs), 1 if on_dev else 0, L.ptr(ploidy_out))
        L.check(L.lib().stp_f2_extract_blocks(self._h, C.byref(r), C.byref(o)))
        t = F2Tensor(f2, vp, bs, P, n_block) if not on_dev else (f2, vp, bs)
        return (t, ploidy_out) if return_ploidy else t

    def extract_streamed(self, records, n_ind: int, sel_rows, pop_offsets, block_id, n_block: int, sink,
                         precision=None, sample_ploidy=None, ploidy="auto", kept_rows=None) -> np.ndarray:
        """stp_f2_extract_streamed: the extraction handed to sink(b0, b1, f2, vpair) in runs of
        finished blocks (numpy views of (b1 - b0) * P * P doubles each, valid during the
        call), so the whole tensor never has to exist. Returns the block sizes."""
        r = self._request(records, n_ind, sel_rows, pop_offsets, block_id, n_block, precision,
                          sample_ploidy, ploidy, kept_rows)
        return self._streamed(lambda cb, bs: L.lib().stp_f2_extract_streamed(self._h, C.byref(r), cb, None, L.ptr(bs)),
                              r.n_pop, n_block, sink)

    def f2_from_qvn_streamed(self, Q, V, N, P: int, block_id, n_block: int, sink, precision=None) -> np.ndarray:
        """stp_f2_from_qvn_streamed (compute_f2_blocks_streamed over dense Q/V/N)."""
        Q, V, N = (np.ascontiguousarray(x, dtype=np.float64) for x in (Q, V, N))
        M = Q.size // P if P > 0 else 0
        bid = _i32(block_id)
        prec = parse_precision(precision)
        return self._streamed(lambda cb, bs: L.lib().stp_f2_from_qvn_streamed(
            self._h, L.ptr(Q), L.ptr(V), L.ptr(N), P, M, L.ptr(bid), n_block, prec, cb, None, L.ptr(bs)),
            P, n_block, sink)

    @staticmethod
    def _streamed(call, P: int, n_block: int, sink) -> np.ndarray:
        err: list[BaseException] = []

        def cb(_user, b0, b1, f2p, vpp):
            try:
                n = (b1 - b0) * P * P
                sink(b0, b1, np.ctypeslib.as_array(f2p, (n,)), np.ctypeslib.as_array(vpp, (n,)))
                return 0
            except BaseException as e:  # the library stops and reports; re-raised below
                err.append(e)
                return 1

        bs = np.zeros(max(n_block, 0), np.int32)
        keep = L.SLAB_SINK(cb)
        st = call(keep, bs)
        if err:
            raise err[0]
        L.check(st)
        return bs

    def extract_batch(self, records, n_ind: int, requests, precision=None, out=None) -> list:
        """Many requests over one panel in one call (stp_f2_extract_batch). requests: a sequence
        of dicts with sel_rows, pop_offsets, block_id, n_block and optionally sample_ploidy /
        ploidy. out: optional list of (f2, vpair) buffers per request (numpy host or torch
        CUDA). Returns one F2Tensor (host outputs) or (f2, vpair, block_sizes) per request."""
        reqs = (L.F2Request * max(len(requests), 1))()
        outs = (L.F2Output * max(len(requests), 1))()
        keep, results = [], []
        for k, q in enumerate(requests):
            r = self._request(records, n_ind, q["sel_rows"], q["pop_offsets"], q["block_id"], int(q["n_block"]),
                              precision, q.get("sample_ploidy"), q.get("ploidy", "auto"))
            reqs[k] = r
            P = r.n_pop
            n = P * P * int(q["n_block"])
            f2, vp = (np.zeros(n), np.zeros(n)) if out is None else out[k]
            bs = np.zeros(max(int(q["n_block"]), 0), np.int32)
            on_dev = _is_torch_cuda(f2)
            outs[k] = L.F2Output(_data_ptr(f2), _data_ptr(vp), L.ptr(bs), 1 if on_dev else 0, None)
            keep.append((r, f2, vp, bs))
            results.append(F2Tensor(f2, vp, bs, P, int(q["n_block"])) if not on_dev else (f2, vp, bs))
        L.check(L.lib().stp_f2_extract_batch(self._h, reqs, len(requests), outs))
        return results

    # -- f-statistics from an F2BlockTensor -----------------------------------------------------
    def fstats(self, f2, vpair, block_sizes, P: int, n_block: int, kind: int, idx, n_stat: int):
        """stp_fstats: (est, var, n_survivors). f2 / vpair flat [P*P*n_block], numpy (host) or
        torch CUDA (device)."""
        on_dev = _is_torch_cuda(f2)
        if not on_dev:
            f2 = np.ascontiguousarray(f2, np.float64)
            vpair = np.ascontiguousarray(vpair, np.float64)
        bs, ix = _i32(block_sizes), _i32(idx)
        if kind == L.FSTAT_F4_LEFT_RIGHT:
            m = max(n_stat - 1, 0) * max(ix.size - n_stat - 1, 0)
        else:
            m = n_stat
        est, var = np.zeros(max(m, 1)), np.zeros(max(m, 1))
        ns = C.c_int32(0)
        L.check(L.lib().stp_fstats(self._h, _data_ptr(f2), _data_ptr(vpair), L.ptr(bs), P, n_block, 1 if on_dev else 0,
                                   kind, L.ptr(ix), ix.size, n_stat, L.ptr(est), L.ptr(var), C.byref(ns)))
        return est[:m], var[:m], int(ns.value)

    def f4(self, t: F2Tensor, quartets):
        """f4(p1, p2; p3, p4) per quartet row with its jackknife variance (est, var, n_survivors)."""
        q = _i32(quartets).reshape(-1, 4)
        return self.fstats(t.f2, t.vpair, t.block_sizes, t.P, t.n_block, L.FSTAT_F4, q.reshape(-1), q.shape[0])

    def f3(self, t: F2Tensor, triples):
        """f3(c; a, b) per triple row (c, a, b)."""
        q = _i32(triples).reshape(-1, 3)
        return self.fstats(t.f2, t.vpair, t.block_sizes, t.P, t.n_block, L.FSTAT_F3, q.reshape(-1), q.shape[0])

    def f4_matrix(self, t: F2Tensor, left, right):
        """qpAdm's f4 matrix: statistic j + nr*i for left[1+i], right[1+j] against left[0],
        right[0]; returned as est, var of shape [nl, nr]."""
        lf, rt = _i32(left), _i32(right)
        est, var, ns = self.fstats(t.f2, t.vpair, t.block_sizes, t.P, t.n_block, L.FSTAT_F4_LEFT_RIGHT,
                                   np.concatenate([lf, rt]), lf.size)
        nl, nr = max(lf.size - 1, 0), max(rt.size - 1, 0)
        return est.reshape(nl, nr), var.reshape(nl, nr), ns

    def last_batch_times(self, n: int) -> np.ndarray:
        """Per-request completion times (ms from the start of the group's device work) of the
        last extract_batch call; NaN for requests that ran on their own."""
        ms = np.zeros(max(n, 0))
        L.check(L.lib().stp_last_batch_times(self._h, L.ptr(ms), n))
        return ms

    def jackknife(self, x, block_sizes, m: int, n_block: int) -> tuple[np.ndarray, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float64)
        bs = _i32(block_sizes)
        est, var = np.zeros(m), np.zeros(m)
        L.check(L.lib().stp_f2_jackknife(self._h, L.ptr(x), L.ptr(bs), m, n_block, L.ptr(est), L.ptr(var)))
        return est, var

    def plan(self, records, n_ind: int, sel_rows, pop_offsets, block_id, n_block: int, precision=None,
             sample_ploidy=None, ploidy="auto", kept_rows=None) -> "Plan":
        return Plan(self, self._request(records, n_ind, sel_rows, pop_offsets, block_id, n_block, precision,
                                        sample_ploidy, ploidy, kept_rows))


class Plan:
    """Device-resident repeated extraction (stp_plan_*): inputs and outputs stay in HBM."""

    def __init__(self, ctx: Context, req: L.F2Request):
        st = C.c_int(0)
        if not ctx._h:
            raise ValueError("the context is closed")
        self._ctx = ctx
        self._h = L.lib().stp_plan_create(ctx._h, C.byref(req), C.byref(st))
        if not self._h:
            raise L.StpError(st.value, L.lib().stp_last_error().decode())
        ctx._plans.add(self)
        self.P = req.n_pop
        self.n_block = req.n_block

    def run(self, records, f2, vpair, stream: int = 0) -> None:
        L.check(L.lib().stp_plan_run(self._h, _data_ptr(records), _data_ptr(f2), _data_ptr(vpair),
                                     stream or None))

    def run_graph(self, records, f2, vpair, stream: int = 0) -> None:
        """The same pass replayed from a CUDA graph (captured on the first call for these
        buffers)."""
        L.check(L.lib().stp_plan_run_graph(self._h, _data_ptr(records), _data_ptr(f2), _data_ptr(vpair),
                                           stream or None))

    @property
    def launches(self) -> int:
        return int(L.lib().stp_plan_launches(self._h))

    def set_per_block_launch(self, on: bool = True) -> None:
        """Comparison form: one contraction launch per jackknife block."""
        L.check(L.lib().stp_plan_set_per_block_launch(self._h, 1 if on else 0))

    def set_timing(self, on: bool = True) -> None:
        L.check(L.lib().stp_plan_set_timing(self._h, 1 if on else 0))

    def last_times(self) -> tuple[float, float]:
        a, b = C.c_float(0), C.c_float(0)
        L.check(L.lib().stp_plan_last_times(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            L.lib().stp_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- the reference's Python surface ---------------------------------------------------------

class F2Blocks:
    """Opaque f2 handle (F2Handle): the host f2 tensor plus population labels."""

    def __init__(self, tensor: F2Tensor, pops: list[str], device: int = 0):
        self._t = tensor
        self._pops = list(pops)
        self._device = device

    @property
    def pops(self) -> list[str]:
        return list(self._pops)

    @property
    def P(self) -> int:
        return self._t.P

    @property
    def n_block(self) -> int:
        return self._t.n_block

    @property
    def block_sizes(self) -> list[int]:
        return [int(x) for x in self._t.block_sizes]

    @property
    def device(self) -> int:
        return self._device

    @property
    def tensor(self) -> F2Tensor:
        return self._t

    def to_numpy(self) -> np.ndarray:
        """f2 as float64, F-contiguous (P, P, n_block). A copy."""
        return np.array(self._t.cube("f2"), order="F", copy=True)

    def vpair_to_numpy(self) -> np.ndarray:
        return np.array(self._t.cube("vpair"), order="F", copy=True)

    def __repr__(self) -> str:
        return f"F2Blocks(P={self.P}, n_block={self.n_block}, device={self.device})"


def read_f2(directory, *, device: int = 0) -> F2Blocks:
    """Loads an f2 directory (f2.bin STPF2BK1 + pops.txt) into an F2Blocks handle."""
    t, pops = read_f2_dir(directory)
    return F2Blocks(t, pops, device)


_CTX: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    if device not in _CTX:
        _CTX[device] = Context(device)
    return _CTX[device]


def extract_f2(prefix, *, pops: list[str], out: str | None = None, device: int = 0, blgsize: float = 0.05,
               maf: float = 0.0, maxmiss: float = 0.0, autosomes_only: bool = True,
               drop_monomorphic: bool = False, transversions_only: bool = False, ploidy: str = "auto",
               strand_mode: str = "drop", precision: str | None = None, tier: str = "host"):
    """Builds an f2_blocks tensor from <prefix>.{geno,snp,ind} on the GPU.

    The P axis is the selection sorted ascending by label (pops.txt order). Returns an
    F2Blocks handle, or writes an STPF2BK1 directory to ``out`` and returns its path.
    SNP filters (maxmiss, maf, monomorphic, autosomes, transversions, strand) are
    applied before the block walk, by the device keep mask over exact counts. tier="disk"
    (with ``out``) streams finished runs of blocks straight into f2.bin, so the tensor is
    never held in host memory (the reference's Disk output tier).
    """
    if tier not in ("host", "disk"):
        raise ValueError("extract_f2: tier must be 'host' or 'disk'")
    if tier == "disk" and out is None:
        raise ValueError("extract_f2: tier='disk' writes to `out`")
    if not pops:
        raise ValueError("extract_f2: pops needs at least one population name")
    if ploidy not in PLOIDY:
        raise ValueError("extract_f2: ploidy must be one of 'auto', '1'/'pseudo', '2'/'diploid'")
    if strand_mode not in ("drop", "keep", "flip"):
        raise ValueError("extract_f2: strand_mode must be one of 'drop', 'keep', 'flip'")
    prec = parse_precision(precision)
    prefix = str(prefix)
    h, rec = read_geno(prefix + ".geno")
    snp = read_snp(prefix + ".snp")
    ind = read_ind(prefix + ".ind")
    if len(ind) < h.n_ind:
        raise ValueError(f"extract_f2: .ind has {len(ind)} rows but .geno has {h.n_ind} individuals")
    if snp.chrom.size < h.n_snp:
        raise ValueError(f"extract_f2: .snp has {snp.chrom.size} rows but the tile spans {h.n_snp} SNPs")
    labels, sel, po = select_pops(ind, pops)
    ctx = context(device)
    M = h.n_snp
    # The keep mask on the device from the exact counts (stp_snp_keep_mask); the kept rows are
    # then read in place by the extraction (no compacted copy of the records). Ploidy is
    # detected on the unfiltered records' first min(1000, M) SNPs, as the reference does
    # (extract_f2_core.cpp:145-166), by both calls.
    keep = ctx.snp_keep_mask(rec, h.n_ind, sel, po, snp.ref[:M], snp.alt[:M], snp.chrom[:M], maf_min=maf,
                             maxmiss=maxmiss, autosomes_only=autosomes_only, drop_monomorphic=drop_monomorphic,
                             transversions_only=transversions_only, strand_mode=strand_mode, ploidy=ploidy)
    idx = np.flatnonzero(keep)
    if idx.size == 0:
        raise ValueError(f"extract_f2: every SNP was filtered out (0 of {h.n_snp} kept) — relax the filters")
    bid, nb = assign_blocks(snp.chrom[idx], snp.genpos[idx], blgsize, snp.physpos[idx])
    if nb <= 0:
        raise ValueError("extract_f2: assign_blocks produced 0 blocks (check blgsize and the .snp genetic positions)")
    kept_rows = None if idx.size == M else idx
    meta = {
        "precision_tag": PRECISION_TAGS.get(prec, ""), "blgsize_cm": blgsize * 100.0,
        "n_snp_total": h.n_snp, "n_snp_kept": int(idx.size),
        "filters": {"maf_min": maf, "maxmiss": maxmiss, "autosomes_only": autosomes_only,
                    "drop_monomorphic": drop_monomorphic, "transversions_only": transversions_only,
                    "strand_mode": strand_mode},
        "pop_selection": "explicit:" + ",".join(pops),
        "geno": prefix + ".geno", "snp": prefix + ".snp", "ind": prefix + ".ind",
    }
    if tier == "disk":
        w = F2DirWriter(out, len(labels), nb, labels, meta)
        bs = ctx.extract_streamed(rec, h.n_ind, sel, po, bid, nb, w.slabs, precision=prec, ploidy=ploidy,
                                  kept_rows=kept_rows)
        w.finish(bs)
        return str(out)
    t = ctx.extract_blocks(rec, h.n_ind, sel, po, bid, nb, precision=prec, ploidy=ploidy, kept_rows=kept_rows)
    if out is None:
        return F2Blocks(t, labels, device)
    write_f2_dir(out, t, labels, meta)
    return str(out)
