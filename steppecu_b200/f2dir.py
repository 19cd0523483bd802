"""STPF2BK1 f2 directories: ``f2.bin`` + ``pops.txt`` + ``meta.json``.

Byte layout of f2.bin (src/device/f2_disk_format.hpp:17-47 and the writer at
src/app/f2_dir_writer.cpp:306-438 in the reference), little-endian:

    0   char[8]  magic "STPF2BK1"
    8   u32      version = 1
    12  u32      dtype = 1 (FP64)
    16  i32      P
    20  i32      n_block
    24  u64      f2_offset          = 64
    32  u64      vpair_offset       = 64 + 8*P*P*n_block
    40  u64      block_sizes_offset = vpair_offset + 8*P*P*n_block
    48  u8[16]   reserved (zero)
    64  f64[P*P*n_block] f2, element (i, j, b) at i + P*j + P*P*b
        f64[P*P*n_block] vpair
        i32[n_block]     block_sizes

meta.json carries provenance and ``f2_cache_id = "sha256:" + sha256(f2.bin)``.
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import struct
from pathlib import Path

import numpy as np

MAGIC = b"STPF2BK1"
VERSION = 1
DTYPE_FP64 = 1
HEADER = struct.Struct("<8sIIiiQQQ16s")
assert HEADER.size == 64


class F2DirError(ValueError):
    """An f2 directory could not be read or written (Status::InvalidConfig)."""


@dataclasses.dataclass
class F2Tensor:
    """F2BlockTensor (include/steppe/fstats.hpp:19-59): f2 and vpair flat FP64
    [P*P*n_block], block_sizes int32 [n_block]."""
    f2: np.ndarray
    vpair: np.ndarray
    block_sizes: np.ndarray
    P: int
    n_block: int

    def f2_at(self, i: int, j: int, b: int) -> float:
        return float(self.f2[i + self.P * j + self.P * self.P * b])

    def vpair_at(self, i: int, j: int, b: int) -> float:
        return float(self.vpair[i + self.P * j + self.P * self.P * b])

    def cube(self, which: str = "f2") -> np.ndarray:
        """(P, P, n_block) F-contiguous view: arr[:, :, b] is slab b."""
        a = self.f2 if which == "f2" else self.vpair
        return a.reshape((self.P, self.P, self.n_block), order="F")


def header_bytes(P: int, n_block: int) -> bytes:
    slab = 8 * P * P * n_block
    return HEADER.pack(MAGIC, VERSION, DTYPE_FP64, P, n_block, 64, 64 + slab, 64 + 2 * slab, b"\0" * 16)


def f2_bin_bytes(t: F2Tensor) -> bytes:
    f2 = np.ascontiguousarray(t.f2, dtype="<f8")
    vp = np.ascontiguousarray(t.vpair, dtype="<f8")
    bs = np.ascontiguousarray(t.block_sizes, dtype="<i4")
    return header_bytes(t.P, t.n_block) + f2.tobytes() + vp.tobytes() + bs.tobytes()


def _sha256_file(path: Path) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 22), b""):
            h.update(chunk)
    return h.hexdigest()


def _jstr(s: str) -> str:
    return json.dumps(s)


def write_f2_dir(directory, t: F2Tensor, pop_labels: list[str], meta: dict | None = None) -> str:
    """Writes f2.bin, pops.txt and meta.json (f2_dir_writer.cpp:306-438). Returns the
    f2_cache_id."""
    meta = dict(meta or {})
    if t.P <= 0 or t.n_block <= 0:
        raise F2DirError(f"write_f2_dir: degenerate f2 tensor (P={t.P} n_block={t.n_block})")
    if len(pop_labels) != t.P:
        raise F2DirError(f"write_f2_dir: pop_labels has {len(pop_labels)} entries but f2 tensor P={t.P}")
    n = t.P * t.P * t.n_block
    if t.f2.size != n or t.vpair.size != n:
        raise F2DirError("write_f2_dir: f2/vpair length mismatch")
    if t.block_sizes.size != t.n_block:
        raise F2DirError("write_f2_dir: block_sizes length mismatch")
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    bin_path = d / "f2.bin"
    with open(bin_path, "wb") as f:
        f.write(f2_bin_bytes(t))
    return _finish_dir(d, t.P, t.n_block, pop_labels, meta)


class F2DirWriter:
    """Writes an STPF2BK1 directory slab by slab (the disk tier of a streamed extraction):
    slabs() takes runs of finished blocks in any order and writes them at their offsets in
    f2.bin, so the P x P x n_block tensor is never held in memory; finish() writes the
    block sizes, pops.txt and meta.json (with the sha256 cache id of the finished f2.bin)."""

    def __init__(self, directory, P: int, n_block: int, pop_labels: list[str], meta: dict | None = None):
        if P <= 0 or n_block <= 0:
            raise F2DirError(f"F2DirWriter: degenerate f2 tensor (P={P} n_block={n_block})")
        if len(pop_labels) != P:
            raise F2DirError(f"F2DirWriter: pop_labels has {len(pop_labels)} entries but P={P}")
        self.d = Path(directory)
        self.d.mkdir(parents=True, exist_ok=True)
        self.P, self.n_block, self.labels, self.meta = P, n_block, list(pop_labels), dict(meta or {})
        self.slab = P * P
        self.f = open(self.d / "f2.bin", "wb")
        self.f.write(header_bytes(P, n_block))
        self.f.truncate(64 + 2 * 8 * self.slab * n_block + 4 * n_block)
        self.written = np.zeros(n_block, bool)

    def slabs(self, b0: int, b1: int, f2: np.ndarray, vpair: np.ndarray) -> None:
        n = (b1 - b0) * self.slab
        for base, a in ((64, f2), (64 + 8 * self.slab * self.n_block, vpair)):
            self.f.seek(base + 8 * self.slab * b0)
            self.f.write(np.ascontiguousarray(a[:n], dtype="<f8").tobytes())
        self.written[b0:b1] = True

    def finish(self, block_sizes: np.ndarray) -> str:
        if not self.written.all():
            raise F2DirError("F2DirWriter: not every block was written")
        bs = np.ascontiguousarray(block_sizes, dtype="<i4")
        if bs.size != self.n_block:
            raise F2DirError("F2DirWriter: block_sizes length mismatch")
        self.f.seek(64 + 2 * 8 * self.slab * self.n_block)
        self.f.write(bs.tobytes())
        self.f.close()
        return _finish_dir(self.d, self.P, self.n_block, self.labels, self.meta)


def _finish_dir(d: Path, P: int, n_block: int, pop_labels: list[str], meta: dict) -> str:
    """pops.txt and meta.json beside a complete f2.bin; returns the f2_cache_id."""
    bin_path = d / "f2.bin"
    cache_id = "sha256:" + _sha256_file(bin_path)
    with open(d / "pops.txt", "w") as f:
        for s in pop_labels:
            f.write(s + "\n")
    pops_sha = "sha256:" + _sha256_file(d / "pops.txt")
    filt = meta.get("filters", {})

    def b(x):
        return "true" if x else "false"

    lines = [
        "{",
        '  "format": "STPF2BK1",',
        '  "meta_schema_version": 1,',
        f'  "steppe_version": {_jstr(meta.get("steppe_version", "stpf2-b200"))},',
        f'  "P": {P},',
        f'  "n_block": {n_block},',
        f'  "precision_tag": {_jstr(meta.get("precision_tag", ""))},',
        f'  "precision_mantissa_bits": {int(meta.get("precision_mantissa_bits", 0))},',
        f'  "blgsize_cm": {meta.get("blgsize_cm", 5)},',
        f'  "n_snp_total": {int(meta.get("n_snp_total", 0))},',
        f'  "n_snp_kept": {int(meta.get("n_snp_kept", 0))},',
        '  "filters": {',
        f'    "maf_min": {filt.get("maf_min", 0)},',
        f'    "maxmiss": {filt.get("maxmiss", 0)},',
        f'    "mind_max_missing": {filt.get("mind_max_missing", 1)},',
        f'    "autosomes_only": {b(filt.get("autosomes_only", True))},',
        f'    "drop_monomorphic": {b(filt.get("drop_monomorphic", False))},',
        f'    "transversions_only": {b(filt.get("transversions_only", False))}',
        "  },",
        f'  "pop_selection": {_jstr(meta.get("pop_selection", ""))},',
        '  "source": {',
        f'    "geno": {_jstr(meta.get("geno", ""))},',
        f'    "snp": {_jstr(meta.get("snp", ""))},',
        f'    "ind": {_jstr(meta.get("ind", ""))},',
        '    "source_hash_computed": false,',
        '    "geno_sha256": "",',
        '    "snp_sha256": "",',
        '    "ind_sha256": ""',
        "  },",
        f'  "pops_sha256": {_jstr(pops_sha)},',
        f'  "f2_cache_id": {_jstr(cache_id)}',
        "}",
    ]
    with open(d / "meta.json", "w") as f:
        f.write("\n".join(lines) + "\n")
    return cache_id


def parse_f2_bin(data: bytes) -> F2Tensor:
    """Parses f2.bin bytes with the reader's checks (src/app/f2_dir_io.cpp:52-156)."""
    if len(data) < 64:
        raise F2DirError("f2.bin is truncated (could not read the 64-byte header)")
    magic, version, dtype, P, nb, off_f2, off_vp, off_bs, _ = HEADER.unpack_from(data, 0)
    if magic != MAGIC:
        raise F2DirError("f2.bin bad magic (expected STPF2BK1)")
    if version != VERSION:
        raise F2DirError(f"f2.bin unsupported version {version}")
    if dtype != DTYPE_FP64:
        raise F2DirError(f"f2.bin unsupported dtype {dtype} (only FP64 is supported)")
    if P <= 0 or nb <= 0:
        raise F2DirError(f"f2.bin degenerate shape P={P} n_block={nb}")
    n = P * P * nb
    if off_f2 + 8 * n > len(data):
        raise F2DirError("f2.bin truncated reading the f2 region")
    if off_vp + 8 * n > len(data):
        raise F2DirError("f2.bin truncated reading the vpair region")
    if off_bs + 4 * nb > len(data):
        raise F2DirError("f2.bin truncated reading the block_sizes trailer")
    f2 = np.frombuffer(data, dtype="<f8", count=n, offset=off_f2).copy()
    vp = np.frombuffer(data, dtype="<f8", count=n, offset=off_vp).copy()
    bs = np.frombuffer(data, dtype="<i4", count=nb, offset=off_bs).copy()
    return F2Tensor(f2, vp, bs, P, nb)


def read_f2_dir(directory) -> tuple[F2Tensor, list[str]]:
    d = Path(directory)
    if not d.is_dir():
        raise F2DirError(f"--f2-dir is not a directory: {d}")
    try:
        data = (d / "f2.bin").read_bytes()
    except OSError as e:
        raise F2DirError(f"cannot open f2.bin ({e.strerror}): {d / 'f2.bin'}") from None
    t = parse_f2_bin(data)
    try:
        labels = [ln.strip() for ln in (d / "pops.txt").read_text().splitlines() if ln.strip()]
    except OSError as e:
        raise F2DirError(f"cannot open pops.txt ({e.strerror})") from None
    if len(labels) != t.P:
        raise F2DirError(f"pops.txt has {len(labels)} labels but f2.bin has P={t.P} populations")
    return t, labels
