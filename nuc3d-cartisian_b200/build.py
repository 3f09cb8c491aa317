"""Build the in-tree CUDA library lib/libnuc3d_b200.so for sm_100a.

    python nuc3d-cartisian_b200/build.py [--force]

Each .cu / .cpp under csrc/ is compiled with nvcc (-gencode arch=compute_100a,
code=sm_100a -lineinfo -O3) in parallel and linked into one shared library
whose C ABI is include/nuc3d_b200.h, and host/nuc3d_run.cpp (the C++ case
driver) into lib/nuc3d_run against it.  The toolchain's g++ links libstdc++
statically; the link hides those symbols (--exclude-libs,ALL) so the library
can share a process with other C++ runtimes (numpy, torch).
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libnuc3d_b200.so"
DRIVER = PKG / "lib" / "nuc3d_run"  # host/nuc3d_run.cpp: the C++ case driver
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# cuFFT (the spectra's transforms) is linked from the toolkit beside nvcc
CUDA_LIB = str(Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "lib64")
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden,-pthread",
              "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale(src: Path, obj: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "nuc3d_b200.h"]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def compile_one(src: Path, force: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    if force or _stale(src, obj):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force), sources()))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs),
               "-Xcompiler", "-static-libstdc++,-pthread", "-Xlinker", "--exclude-libs,ALL",
               "-cudart", "static", "-lcufft", "-Xlinker", "-rpath," + CUDA_LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, LIB)
    build_driver(force)
    if verbose:
        print(f"built {LIB}")
    return LIB


def build_driver(force: bool = False) -> Path:
    """The C++ case driver, linked against the library (C ABI only)."""
    src = PKG / "host" / "nuc3d_run.cpp"
    if (force or not DRIVER.exists() or src.stat().st_mtime > DRIVER.stat().st_mtime
            or LIB.stat().st_mtime > DRIVER.stat().st_mtime):
        cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
        cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-I", str(ROOT / "include"), str(src),
               "-L", str(LIB.parent), "-lnuc3d_b200", "-Wl,-rpath,$ORIGIN", "-o", str(DRIVER)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed:\n{r.stderr}")
    return DRIVER


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    try:
        build(force=a.force, verbose=True)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
