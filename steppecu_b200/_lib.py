"""ctypes binding of libstpf2.so (include/stpf2.h).

The library is the product path; there is no CPU fallback. Loading fails loudly if the
shared library has not been built.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libstpf2.so"

STP_OK = 0
STP_DEVICE_OOM = 1
STP_INVALID_CONFIG = 5
STP_INVALID_ARGUMENT = 100
STP_RUNTIME_ERROR = 101
STP_CUDA_ERROR = 102
STP_NO_DEVICE = 103
STP_DEVICE_TIMEOUT = 104

STATUS_NAMES = {
    STP_OK: "ok",
    STP_DEVICE_OOM: "device_oom",
    STP_INVALID_CONFIG: "invalid_config",
    STP_INVALID_ARGUMENT: "invalid_argument",
    STP_RUNTIME_ERROR: "runtime_error",
    STP_CUDA_ERROR: "cuda_error",
    STP_NO_DEVICE: "no_device",
    STP_DEVICE_TIMEOUT: "device_timeout",
}

PREC_FP32_SIMT = 0
PREC_SPLIT_BF16 = 1
PREC_SPLIT_F16 = 2
PREC_SPLIT_F16_FINE = 3
PREC_FIXED_I8 = 4
FSTAT_F4 = 0
FSTAT_F3 = 1
FSTAT_F4_LEFT_RIGHT = 2

PLOIDY_AUTO = 0
PLOIDY_PSEUDO = 1
PLOIDY_DIPLOID = 2


class StpError(RuntimeError):
    """A libstpf2 call failed; ``status`` is the stp_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class GenoView(C.Structure):
    _fields_ = [
        ("records", C.c_void_p),
        ("bytes_per_record", C.c_uint64),
        ("pitch", C.c_uint64),
        ("n_snp", C.c_int64),
        ("n_ind", C.c_int64),
        ("on_device", C.c_int32),
    ]


class F2Request(C.Structure):
    _fields_ = [
        ("geno", GenoView),
        ("sel_rows", C.c_void_p),
        ("pop_offsets", C.c_void_p),
        ("n_pop", C.c_int32),
        ("sample_ploidy", C.c_void_p),
        ("ploidy_mode", C.c_int32),
        ("block_id", C.c_void_p),
        ("n_block", C.c_int32),
        ("precision", C.c_int32),
        ("kept_rows", C.c_void_p),
        ("n_kept", C.c_int64),
    ]


class F2Output(C.Structure):
    _fields_ = [
        ("f2", C.c_void_p),
        ("vpair", C.c_void_p),
        ("block_sizes", C.c_void_p),
        ("on_device", C.c_int32),
        ("ploidy_out", C.c_void_p),
    ]


class SnpFilter(C.Structure):
    _fields_ = [
        ("maf_min", C.c_double),
        ("maxmiss", C.c_double),
        ("autosomes_only", C.c_int32),
        ("drop_monomorphic", C.c_int32),
        ("transversions_only", C.c_int32),
        ("strand_mode", C.c_int32),
    ]


STRAND_DROP, STRAND_KEEP, STRAND_FLIP = 0, 1, 2

# stp_slab_sink: int (*)(void* user, int32_t b0, int32_t b1, const double* f2, const double* vpair)
SLAB_SINK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double))

# Every symbol include/stpf2.h declares, with its ctypes signature (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "stp_abi_version": (C.c_int, []),
    "stp_last_error": (C.c_char_p, []),
    "stp_create": (_P, [C.c_int, C.POINTER(C.c_int)]),
    "stp_destroy": (None, [_P]),
    "stp_launch_count": (C.c_uint64, [_P]),
    "stp_set_wait_bounds": (C.c_int, [_P, C.c_uint64, C.c_int64]),
    "stp_set_tile_classes": (C.c_int, [_P, C.c_uint32]),
    "stp_detect_ploidy": (C.c_int, [_P, C.POINTER(GenoView), _P, C.c_int64, _P]),
    "stp_detect_ploidy_tile": (C.c_int, [_P, _P, C.c_uint64, C.c_int64, C.c_int64, C.c_int32, _P]),
    "stp_decode_counts": (C.c_int, [_P, C.POINTER(GenoView), _P, _P, C.c_int32, _P, C.c_int32, _P, _P]),
    "stp_decode_counts_noalloc": (C.c_int, [_P, C.POINTER(GenoView), _P, _P, C.c_int32, _P, C.c_int32, _P, _P, _P]),
    "stp_f2_from_qvn_device": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int64, _P, C.c_int32, C.c_int32, C.c_int32,
                                         _P, _P, _P]),
    "stp_f2_from_qvn_streamed": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int64, _P, C.c_int32, C.c_int32,
                                           SLAB_SINK, _P, _P]),
    "stp_f2_extract_streamed": (C.c_int, [_P, C.POINTER(F2Request), SLAB_SINK, _P, _P]),
    "stp_canonical_to_records": (C.c_int, [_P, _P, C.c_uint64, C.c_int64, C.c_int64, C.c_int32, _P, C.c_uint64]),
    "stp_snp_keep_mask": (C.c_int, [_P, C.POINTER(GenoView), _P, _P, C.c_int32, _P, C.c_int32, _P, _P, _P,
                                    C.POINTER(SnpFilter), _P, C.POINTER(C.c_int64), _P]),
    "stp_decode_af_compact_filter": (C.c_int, [_P, _P, C.c_uint64, C.c_int64, C.c_int64, _P, C.c_int32, _P, C.c_int32,
                                               C.c_int32, _P, _P, _P, C.POINTER(SnpFilter), C.c_double, _P,
                                               C.POINTER(C.c_int64), _P, _P, _P, C.c_int32]),
    "stp_decode_af": (C.c_int, [_P, _P, C.c_uint64, C.c_int64, C.c_int64, _P, C.c_int32, _P, C.c_int32,
                                C.c_int32, C.c_int32, _P, _P, _P]),
    "stp_f2_from_qvn": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int64, _P, C.c_int32, C.c_int32, _P, _P, _P]),
    "stp_f2_extract_blocks": (C.c_int, [_P, C.POINTER(F2Request), C.POINTER(F2Output)]),
    "stp_f2_extract_batch": (C.c_int, [_P, C.POINTER(F2Request), C.c_int32, C.POINTER(F2Output)]),
    "stp_last_batch_times": (C.c_int, [_P, _P, C.c_int32]),
    "stp_fstats": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int64, C.c_int64,
                             _P, _P, _P]),
    "stp_f2_jackknife": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int32, _P, _P]),
    "stp_plan_create": (_P, [_P, C.POINTER(F2Request), C.POINTER(C.c_int)]),
    "stp_plan_run": (C.c_int, [_P, _P, _P, _P, _P]),
    "stp_plan_run_graph": (C.c_int, [_P, _P, _P, _P, _P]),
    "stp_plan_set_per_block_launch": (C.c_int, [_P, C.c_int32]),
    "stp_plan_launches": (C.c_int32, [_P]),
    "stp_plan_set_timing": (C.c_int, [_P, C.c_int32]),
    "stp_plan_last_times": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "stp_plan_destroy": (None, [_P]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded libstpf2.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
            )
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != STP_OK:
        raise StpError(status, lib().stp_last_error().decode())


def ptr(a: np.ndarray | None) -> int | None:
    """Host pointer of a C-contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"], "array must be contiguous"
    return a.ctypes.data
