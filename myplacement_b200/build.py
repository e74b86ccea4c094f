"""Builds libmpgp.so in-tree: nvcc for sm_100a, one shared library with a C ABI.

    python -m myplacement_b200.build        # incremental
    python -m myplacement_b200.build --force

Every .cu/.cpp under csrc/ is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked against
the CUDA runtime only (no torch, no cuFFT/cuBLAS).  Host files are compiled
with -ffp-contract=off: the host setup must be bit-identical to the reference's.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
CSRC = PACKAGE / "csrc"
BUILD = PACKAGE / "_build"
TARGET = PACKAGE / "libmpgp.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return path


def _sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def _headers_mtime() -> float:
    headers = [*CSRC.glob("*.cuh"), *CSRC.glob("*.hpp"), REPO / "include" / "mpgp.h"]
    return max((h.stat().st_mtime for h in headers if h.exists()), default=0.0)


# Kernels that have a batched twin (one body inlined into a plain and a batched
# kernel) are compiled without fused multiply-add contraction: every product and
# sum is rounded on its own, so the two inlined copies compute the same bits
# whatever the compiler does around them, and a batched placement equals its plain
# run.  The detailed placer keeps contraction: its order choice must round as the
# reference backend's compiled arithmetic does.
UNFUSED = {"batch.cu", "density.cu", "dct_tc.cu", "engine.cu", "gather.cu", "wirelength.cu"}


def _compile(source: Path, force: bool, headers_mtime: float, verbose_ptxas: bool) -> Path:
    obj = BUILD / (source.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime > max(source.stat().st_mtime, headers_mtime):
        return obj
    cmd = [
        _nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
        f"-I{REPO / 'include'}", f"-I{CSRC}", "-c", str(source), "-o", str(obj),
    ]
    if source.suffix == ".cu":
        cmd.insert(1, "--expt-relaxed-constexpr")
        if source.name in UNFUSED:
            cmd.insert(1, "-fmad=false")
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{result.stdout}\n{result.stderr}")
    if verbose_ptxas and result.stderr:
        print(f"== {source.name}\n{result.stderr}")
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    headers_mtime = _headers_mtime()
    sources = _sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        objects = list(pool.map(lambda s: _compile(s, force, headers_mtime, verbose_ptxas), sources))
    newest = max(o.stat().st_mtime for o in objects)
    if force or not TARGET.exists() or TARGET.stat().st_mtime < newest:
        cmd = [_nvcc(), "-shared", *ARCH, "-o", str(TARGET), *map(str, objects), "-lcudart"]
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"link failed:\n{result.stdout}\n{result.stderr}")
    return TARGET


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill reports")
    args = parser.parse_args()
    print(build(force=args.force, verbose_ptxas=args.ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
