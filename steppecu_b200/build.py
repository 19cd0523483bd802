"""Build recipe for the native parts of steppecu_b200.

- ``libstpf2.so``: every CUDA source in ``csrc/`` compiled for sm_100a (B200) only (and the
  host-only ``.cpp`` sources there), with the CUDA runtime linked statically, so the library needs nothing from torch.
- ``oracle/``: the CPU checkers (``make -C oracle``); the reference's own CpuBackend is
  built there too when the reference sources are present.

Objects go to ``_build/`` at the repository root; the shared libraries are written in-tree
so they travel with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libstpf2.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_lib(verbose: bool = False, extra: list[str] | None = None) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "stpf2.h"]
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))  # .cpp: host-only sources
    flags = NVFLAGS + (extra or [])

    def compile_one(src: Path) -> Path:
        obj = BUILD / (src.stem + ".o")
        if _stale(obj, [src] + headers):
            cmd = [nvcc, *flags, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    if _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def build_oracle(verbose: bool = False) -> None:
    cmd = ["make", "-s", "-C", str(ROOT / "oracle")]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_all(verbose: bool = False) -> None:
    build_lib(verbose)
    build_oracle(verbose)


if __name__ == "__main__":
    build_all(verbose=True)
