"""Builds restir_b200/librestir_gpu.so in the source tree.

CUDA sources (csrc/*.cu) are compiled for sm_100a only, as relocatable
device code (they share the device status word), with --fmad=false and IEEE
division and square root (include/restir_numeric.h); host sources
(host/*.cpp) with -ffp-contract=off. Objects go to restir_b200/_build/ and are
rebuilt when a source or header is newer. Run as `python -m restir_b200.build`.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
HOST = PACKAGE / "host"
BUILD = PACKAGE / "_build"
LIBRARY = PACKAGE / "librestir_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-rdc=true",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
    "-I", str(ROOT / "include"),
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             "-I", str(ROOT / "include"), "-I", "/usr/local/cuda/include"]


def _nvcc() -> str:
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(home) / "bin" / "nvcc"
    return str(candidate) if candidate.exists() else (shutil.which("nvcc") or "nvcc")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(HOST.glob("*.h")) + sorted((ROOT / "include").glob("*.h"))


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    stamp = target.stat().st_mtime
    return any(s.stat().st_mtime > stamp for s in sources)


def _run(command: list[str]) -> None:
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(command) + "\n" + result.stdout + result.stderr)


FAST_LIBRARY = PACKAGE / "librestir_gpu_fast.so"
CHECKED_LIBRARY = PACKAGE / "librestir_gpu_checked.so"


def build(verbose: bool = False, defines: list[str] | None = None, library: Path = LIBRARY,
          objects_dir: Path = BUILD, contract: bool = False) -> Path:
    """Compiles stale objects and links the library. defines: extra -D macros for
    the CUDA sources (tuning knobs such as RESTIR_GI_TEMPORAL_MIN_BLOCKS=4),
    built into their own objects_dir and library. contract: the kernels with
    FMA contraction (--fmad=true), a measurement variant that leaves the
    parity conventions of include/restir_numeric.h (its results differ from
    the oracle's in the last bits)."""
    objects_dir = Path(objects_dir)
    objects_dir.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    extra = [f"-D{d}" for d in (defines or [])]
    nvcc_flags = [("--fmad=true" if f == "--fmad=false" else f) for f in NVCC_FLAGS] if contract else NVCC_FLAGS
    jobs = []
    objects = []
    for source in sorted(CSRC.glob("*.cu")):
        obj = objects_dir / (source.stem + ".cu.o")
        objects.append(obj)
        if _stale(obj, [source] + headers):
            jobs.append([nvcc] + nvcc_flags + extra + ["-c", str(source), "-o", str(obj)])
    for source in sorted(HOST.glob("*.cpp")):
        obj = objects_dir / (source.stem + ".cpp.o")
        objects.append(obj)
        if _stale(obj, [source] + headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", str(source), "-o", str(obj)])
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        for command in jobs:
            if verbose:
                print(" ".join(command), file=sys.stderr)
        list(pool.map(_run, jobs))
    library = Path(library)
    library.parent.mkdir(parents=True, exist_ok=True)
    if jobs or _stale(library, objects):
        _run([nvcc] + ARCH + ["-shared", "-rdc=true", "-Xcompiler", "-fPIC"] + [str(o) for o in objects]
             + ["-o", str(library), "-lcudart"])
    return library


if __name__ == "__main__":
    if "--checks" in sys.argv:
        print(build(verbose="-v" in sys.argv, defines=["RESTIR_CHECKS=1"], library=CHECKED_LIBRARY,
                    objects_dir=BUILD.parent / "_build_checked"))
    elif "--contract" in sys.argv:
        print(build(verbose="-v" in sys.argv, library=FAST_LIBRARY, objects_dir=BUILD.parent / "_build_contract",
                    contract=True))
    else:
        print(build(verbose="-v" in sys.argv))
