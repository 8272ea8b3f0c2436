"""Build recipe for libwarpstate_b200.so (sm_100a) and the oracle.

Compiles every CUDA source with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and the host C++
with g++, then links one shared library in the package directory so that it
travels with the repository snapshot.  Incremental: an object is rebuilt only
when its source or a header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libwarpstate_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-Xptxas", "-v"]


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))


def _stale(src: Path, obj: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in _headers())


def _compile(src: Path) -> tuple[Path, str]:
    obj = BUILD / (src.name + ".o")
    log = ""
    if _stale(src, obj):
        if src.suffix == ".cu":
            cmd = [NVCC, *NVFLAGS, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++", *CXXFLAGS, "-I", "/usr/local/cuda/include", "-I", str(ROOT / "include"),
                   "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        log = r.stdout + r.stderr
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {src.name}\n{log}")
    return obj, log


def build_library(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(_compile, sources))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed\n" + r.stdout + r.stderr)
    return LIB


def build_oracle() -> Path:
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed\n" + r.stdout + r.stderr)
    return ROOT / "oracle" / "liboracle.so"


def build_workloads() -> Path:
    r = subprocess.run(["make", "-s", "-C", str(ROOT / "workloads")], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("workload generator build failed\n" + r.stdout + r.stderr)
    return ROOT / "workloads" / "libworkloads.so"


if __name__ == "__main__":
    print(build_library(verbose="-v" in sys.argv))
    print(build_oracle())
    print(build_workloads())
