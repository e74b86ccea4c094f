"""Build recipe for the test oracle (test infrastructure, not the product).

Outputs go to ``oracle/_ref/`` (git-ignored; the built ``.so`` files travel to
the GPU host with the rest of the working tree):

``libref_cpu.so``
    The reference's own CPU global-placement path, compiled from the unmodified
    reference sources, with ``oracle/fftw_shim`` standing in for FFTW3 and
    ``oracle/ref_capi.cpp`` exposing a C ABI.
``libref_cuda.so``
    The same, with the reference CUDA backends
    (src/placement/cuda/CudaPlacementBackend.cu and
    CudaDetailedPlacementBackend.cu) compiled for sm_100a in place of the stubs,
    and ``oracle/policy_override`` replacing the shared-server GPU allow-list so
    device 0 is accepted.
``libref_dropin.so``
    The reference controller linked against this project's drop-in adapters
    and ``libmpgp.so``: myplacement_b200/adapter/mpgp_placement_backend.cpp in
    place of the CUDA backend (the reference's own AdaptiveGlobalPlacer
    driving the B200 engine through the C ABI) and
    myplacement_b200/adapter/mpgp_bookshelf_parser.cpp in place of
    src/io/BookshelfParser.cpp (the reference's BookshelfParser API over the
    native reader), and myplacement_b200/adapter/mpgp_detailed_placement_backend.cpp
    in place of the CUDA detailed-placement backend (DetailedPlacer::run with the
    cuda backend over the engine's window reorder).

``oracle/liboracle.so`` is the project's own C restatement (fixed-point density).

The reference tree is only read; it is compiled where it lies.  When it is
absent (the GPU host), building is skipped and the prebuilt files are used.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

ORACLE = Path(__file__).resolve().parent
REPO = ORACLE.parent
REF_ROOT = Path(os.environ.get("MPGP_REFERENCE_ROOT", "/root/reference"))
OUT = ORACLE / "_ref"
OBJ = OUT / "obj"

CPU_SOURCES = [
    "src/io/BookshelfParser.cpp",
    "src/model/PlacementDatabase.cpp",
    "src/metrics/Metrics.cpp",
    "src/metrics/Rudy.cpp",
    "src/placement/GlobalPlacementSupport.cpp",
    "src/placement/ElectrostaticField.cpp",
    "src/placement/GlobalPlacer.cpp",
    "src/placement/LegacyGlobalPlacer.cpp",
    "src/placement/DetailedPlacer.cpp",
]
STUB_SOURCES = ["src/placement/CudaPlacementBackendStub.cpp", "src/placement/CudaDetailedPlacementBackendStub.cpp"]
CUDA_SOURCES = ["src/placement/cuda/CudaPlacementBackend.cu", "src/placement/cuda/CudaDetailedPlacementBackend.cu"]
ADAPTERS = ["mpgp_placement_backend.cpp", "mpgp_bookshelf_parser.cpp", "mpgp_detailed_placement_backend.cpp"]

CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off"]


def _includes() -> list[str]:
    return [
        f"-I{ORACLE / 'policy_override'}",
        f"-I{REF_ROOT / 'include'}",
        f"-I{REF_ROOT / 'src' / 'placement'}",
        f"-I{ORACLE / 'fftw_shim'}",
        f"-I{REPO / 'include'}",
    ]


def _run(cmd: list[str]) -> None:
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"oracle build failed: {' '.join(cmd)}\n{result.stdout}\n{result.stderr}")


def _object(source: Path, tag: str) -> Path:
    return OBJ / f"{tag}_{source.stem}.o"


def _compile_cxx(source: Path, tag: str) -> Path:
    target = _object(source, tag)
    if target.exists() and target.stat().st_mtime > source.stat().st_mtime:
        return target
    _run(["g++", *CXXFLAGS, *_includes(), "-c", str(source), "-o", str(target)])
    return target


def _compile_cuda(source: Path, tag: str) -> Path:
    target = _object(source, tag)
    if target.exists() and target.stat().st_mtime > source.stat().st_mtime:
        return target
    _run([
        "nvcc", "-std=c++17", "-O2", "-Xcompiler", "-fPIC",
        "-gencode", "arch=compute_100a,code=sm_100a", *_includes(), "-c", str(source), "-o", str(target),
    ])
    return target


def reference_available() -> bool:
    return (REF_ROOT / "src" / "placement" / "AdaptiveGlobalPlacer.cpp").is_file()


def build_oracle_c() -> Path:
    """Compile the project's own C restatement (oracle/density_fixed.c)."""
    target = ORACLE / "liboracle.so"
    source = ORACLE / "density_fixed.c"
    if target.exists() and target.stat().st_mtime > source.stat().st_mtime:
        return target
    _run(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
          str(source), "-o", str(target), "-lm"])
    return target


def build_reference(dropin: bool = True, cuda: bool = True) -> list[Path]:
    """Compile the reference CPU path (and optionally its CUDA backend and the drop-in)."""
    if not reference_available():
        return []
    OBJ.mkdir(parents=True, exist_ok=True)
    shim = ORACLE / "fftw_shim" / "fftw_shim.cpp"
    capi = ORACLE / "ref_capi.cpp"
    common_jobs = [REF_ROOT / s for s in CPU_SOURCES] + [shim, capi]
    adapters = [REPO / "myplacement_b200" / "adapter" / name for name in ADAPTERS]
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        futures = [pool.submit(_compile_cxx, s, "ref") for s in common_jobs]
        stub_futures = [pool.submit(_compile_cxx, REF_ROOT / s, "ref") for s in STUB_SOURCES]
        cuda_futures = [pool.submit(_compile_cuda, REF_ROOT / s, "ref") for s in CUDA_SOURCES] if cuda else []
        adapter_futures = [pool.submit(_compile_cxx, a, "dropin") for a in adapters] if dropin else []
        common = [f.result() for f in futures]
        stubs = [f.result() for f in stub_futures]
        cuda_objects = [f.result() for f in cuda_futures]
        adapter_objects = [f.result() for f in adapter_futures]

    built = []
    cpu_lib = OUT / "libref_cpu.so"
    _run(["g++", "-shared", "-o", str(cpu_lib), *map(str, common), *map(str, stubs)])
    built.append(cpu_lib)
    if cuda_objects:
        cuda_lib = OUT / "libref_cuda.so"
        cuda_home = Path(shutil.which("nvcc")).resolve().parent.parent
        _run(["g++", "-shared", "-o", str(cuda_lib), *map(str, common), *map(str, cuda_objects),
              f"-L{cuda_home / 'lib64'}", "-lcufft", "-lcudart", f"-Wl,-rpath,{cuda_home / 'lib64'}"])
        built.append(cuda_lib)
    if adapter_objects:
        engine = REPO / "myplacement_b200" / "libmpgp.so"
        if engine.exists():
            # The reference's BookShelf reader gives way to the adapter's.
            reader = _object(REF_ROOT / CPU_SOURCES[0], "ref")
            kept = [o for o in common if o != reader]
            dropin_lib = OUT / "libref_dropin.so"
            _run(["g++", "-shared", "-o", str(dropin_lib), *map(str, kept), *map(str, adapter_objects),
                  f"-L{engine.parent}", "-lmpgp", "-Wl,-rpath,$ORIGIN/../../myplacement_b200"])
            built.append(dropin_lib)
    return built


def main() -> int:
    build_oracle_c()
    built = build_reference()
    for path in built:
        print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
