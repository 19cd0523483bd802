"""steppecu_b200 — B200-native (sm_100a) f2 block-tensor extraction.

A drop-in for the extract-f2 path of Steppe (suzuenhasa/steppecu): 2-bit
PACKEDANCESTRYMAP genotypes -> exact per-population allele counts -> per-jackknife-block
bias-corrected f2 means and both-present SNP counts (the FP64 F2BlockTensor / STPF2BK1
output). The compute lives in libstpf2.so (CUDA for sm_100a, C ABI in include/stpf2.h).
"""
from ._lib import StpError
from .api import Context, F2Blocks, Plan, context, extract_f2, parse_precision, read_f2
from .blocks import assign_blocks, block_ranges
from .f2dir import F2Tensor, read_f2_dir, write_f2_dir

__all__ = [
    "Context", "F2Blocks", "F2Tensor", "Plan", "StpError", "assign_blocks", "block_ranges", "context",
    "extract_f2", "parse_precision", "read_f2", "read_f2_dir", "write_f2_dir",
]
