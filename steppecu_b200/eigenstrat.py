"""PACKEDANCESTRYMAP genotype triples (.geno / .snp / .ind) on the host.

Follows the reference's io leaf: the 48-byte text header ``GENO nind nsnp ...``
(parse_geno_header, src/io/eigenstrat_format.cpp:17-85), records of max(48, ceil(nind/4))
bytes, the header occupying one record, SNP-major, four 2-bit codes per byte MSB-first.
"""
from __future__ import annotations

import dataclasses
import re
from pathlib import Path

import numpy as np

HEADER_BYTES = 48
CHROM_X, CHROM_Y, CHROM_MT = 23, 24, 90  # src/io/eigenstrat_format.hpp


class GenoFormatError(ValueError):
    pass


@dataclasses.dataclass
class GenoHeader:
    n_ind: int
    n_snp: int
    bytes_per_record: int
    header_bytes: int


def parse_geno_header(head: bytes) -> GenoHeader:
    text = head[:HEADER_BYTES].split(b"\0", 1)[0].decode("ascii", "replace")
    parts = text.split()
    if not parts or parts[0] != "GENO":
        if parts and parts[0] == "TGENO":
            raise GenoFormatError("TGENO (individual-major) files are not a PACKEDANCESTRYMAP .geno")
        raise GenoFormatError("not a PACKEDANCESTRYMAP .geno (missing GENO magic)")
    nums = re.findall(r"\d+", text[len(parts[0]):])
    if len(nums) < 2:
        raise GenoFormatError("GENO header lacks the individual/SNP counts")
    n_ind, n_snp = int(nums[0]), int(nums[1])
    bpr = max(HEADER_BYTES, (n_ind + 3) // 4)
    return GenoHeader(n_ind, n_snp, bpr, bpr)


def read_geno(path) -> tuple[GenoHeader, np.ndarray]:
    """Returns the header and the SNP-major records as a read-only memory map
    [n_snp, bytes_per_record] uint8."""
    path = Path(path)
    with open(path, "rb") as f:
        head = f.read(HEADER_BYTES)
    h = parse_geno_header(head)
    size = path.stat().st_size
    need = h.header_bytes + h.n_snp * h.bytes_per_record
    if size < need:
        raise GenoFormatError(f"{path}: short file ({size} bytes, header says {need})")
    rec = np.memmap(path, dtype=np.uint8, mode="r", offset=h.header_bytes,
                    shape=(h.n_snp, h.bytes_per_record))
    return h, rec


def _chrom_code(tok: str) -> int:
    t = tok.strip()
    if t.lower().startswith("chr"):
        t = t[3:]
    if t.isdigit():
        return int(t)
    u = t.upper()
    if u == "X":
        return CHROM_X
    if u == "Y":
        return CHROM_Y
    if u in ("MT", "M"):
        return CHROM_MT
    return -1


@dataclasses.dataclass
class SnpTable:
    ids: list[str]
    chrom: np.ndarray
    genpos: np.ndarray     # Morgans
    physpos: np.ndarray
    ref: np.ndarray        # uint8 characters
    alt: np.ndarray


def read_snp(path) -> SnpTable:
    ids, chrom, gp, pp, ref, alt = [], [], [], [], [], []
    with open(path) as f:
        for ln in f:
            t = ln.split()
            if len(t) < 3 or t[0].startswith("#"):
                continue
            ids.append(t[0])
            chrom.append(_chrom_code(t[1]))
            gp.append(float(t[2]))
            pp.append(float(t[3]) if len(t) > 3 else 0.0)
            ref.append(ord(t[4][0]) if len(t) > 4 else ord("N"))
            alt.append(ord(t[5][0]) if len(t) > 5 else ord("N"))
    return SnpTable(ids, np.asarray(chrom, np.int32), np.asarray(gp, np.float64), np.asarray(pp, np.float64),
                    np.asarray(ref, np.uint8), np.asarray(alt, np.uint8))


def read_ind(path) -> list[str]:
    """Population label of every .ind row (third column)."""
    out = []
    with open(path) as f:
        for ln in f:
            t = ln.split()
            if len(t) >= 3:
                out.append(t[2])
            elif t:
                out.append("")
    return out


def select_pops(ind_labels: list[str], pops: list[str]) -> tuple[list[str], np.ndarray, np.ndarray]:
    """Explicit population selection: the P axis is the selection sorted ascending by
    label (pops.txt order); within a population, file order. Returns (labels, sel_rows,
    pop_offsets). Raises KeyError for a population with no individuals."""
    want = sorted(set(pops))
    rows_of: dict[str, list[int]] = {p: [] for p in want}
    for r, lab in enumerate(ind_labels):
        if lab in rows_of:
            rows_of[lab].append(r)
    missing = [p for p in want if not rows_of[p]]
    if missing:
        raise KeyError(f"population(s) not found in .ind: {', '.join(missing)}")
    sel, offs = [], [0]
    for p in want:
        sel.extend(rows_of[p])
        offs.append(len(sel))
    return want, np.asarray(sel, np.int64), np.asarray(offs, np.int64)
