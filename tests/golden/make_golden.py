"""Regenerates the committed STPF2BK1 golden fixtures from the reference's own example.

Source: docs/examples/f2_9pop/{f2.bin, pops.txt, meta.json} in the reference (a real
`steppe extract-f2` output, P = 9, 710 blocks). Written here:

- f2_9pop_header.bin   the file's 64-byte header, verbatim;
- f2_9pop_head.npz     f2 / vpair / block_sizes of the first HEAD_BLOCKS blocks, the full
                       block_sizes trailer, P, n_block, and the sha256 of the whole f2.bin
                       and of pops.txt (both also quoted in the example's meta.json);
- f2_9pop_pops.txt     the population labels in P-axis order.

Run from the repository root: python tests/golden/make_golden.py [reference_root]
(default: $STEPPE_REFERENCE_ROOT).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HEAD_BLOCKS = 12
HERE = Path(__file__).resolve().parent


def main(ref_root: str = "") -> None:
    ref_root = ref_root or os.environ.get("STEPPE_REFERENCE_ROOT", "")
    if not ref_root:
        raise SystemExit("give the reference checkout as an argument or in STEPPE_REFERENCE_ROOT")
    ex = Path(ref_root) / "docs" / "examples" / "f2_9pop"
    data = (ex / "f2.bin").read_bytes()
    pops = (ex / "pops.txt").read_bytes()
    meta = json.loads((ex / "meta.json").read_text())
    P = int(np.frombuffer(data, "<i4", 1, 16)[0])
    nb = int(np.frombuffer(data, "<i4", 1, 20)[0])
    off_f2, off_vp, off_bs = (int(x) for x in np.frombuffer(data, "<u8", 3, 24))
    slab = P * P
    f2 = np.frombuffer(data, "<f8", slab * nb, off_f2)
    vp = np.frombuffer(data, "<f8", slab * nb, off_vp)
    bs = np.frombuffer(data, "<i4", nb, off_bs)
    (HERE / "f2_9pop_header.bin").write_bytes(data[:64])
    (HERE / "f2_9pop_pops.txt").write_bytes(pops)
    np.savez_compressed(
        HERE / "f2_9pop_head.npz",
        f2=f2[: slab * HEAD_BLOCKS].copy(),
        vpair=vp[: slab * HEAD_BLOCKS].copy(),
        block_sizes_head=bs[:HEAD_BLOCKS].copy(),
        block_sizes_all=bs.copy(),
        P=P,
        n_block=nb,
        file_sha256=hashlib.sha256(data).hexdigest(),
        file_size=len(data),
        pops_sha256=hashlib.sha256(pops).hexdigest(),
        meta_f2_cache_id=meta["f2_cache_id"],
        meta_pops_sha256=meta["pops_sha256"],
    )
    print(f"wrote fixtures: P={P} n_block={nb} head={HEAD_BLOCKS}")


if __name__ == "__main__":
    main(*sys.argv[1:])
