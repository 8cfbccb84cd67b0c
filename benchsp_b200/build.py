"""Builds libbspmv.so in-tree (benchsp_b200/lib/) with nvcc for sm_100a.

    python -m benchsp_b200.build          # incremental
    python -m benchsp_b200.build --force  # rebuild everything

CUDA sources compile with -gencode arch=compute_100a,code=sm_100a; host
sources (generators, the C++ host API) with g++.  The CUDA runtime is linked
statically so the library does not depend on which libcudart a host process
(for example PyTorch) has already loaded.
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
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "lib" / "libbspmv.so"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.environ.get("NVCC", str(Path(CUDA_HOME) / "bin" / "nvcc"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fopenmp",
              "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-fopenmp", "-Wall", f"-I{INCLUDE}", f"-I{CSRC}",
             f"-I{CUDA_HOME}/include"]


def _sources() -> list[Path]:
    return sorted([*CSRC.glob("*.cu"), *CSRC.glob("*.cpp")])


def _headers() -> list[Path]:
    return sorted([*CSRC.glob("*.cuh"), *CSRC.glob("*.h"), *INCLUDE.glob("*.h")])


def _compile(src: Path, obj: Path) -> None:
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles changed sources and links benchsp_b200/lib/libbspmv.so."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime)
        if stale:
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
            futs = {ex.submit(_compile, s, o): s for s, o in jobs}
            for f in cf.as_completed(futs):
                f.result()
                if verbose:
                    print("compiled", futs[f].name, file=sys.stderr)
    newest = max(o.stat().st_mtime for o in objs)
    if force or jobs or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp",
               "-Xlinker", "--exclude-libs,ALL", "-Xlinker", "-Bsymbolic"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    _build_compat(force)
    return LIB


COMPAT_SRC = PKG / "compat"
COMPAT_LIB = PKG / "lib" / "libbspmv_compat.so"


def _build_compat(force: bool = False) -> Path:
    """Links libbspmv_compat.so: the reference's C++ operator names
    (include/benchsp_compat.hpp) over libbspmv's C ABI, plus the cuSPARSE
    comparison wrappers.  Host code only (g++)."""
    srcs = sorted(COMPAT_SRC.glob("*.cpp"))
    deps = [*srcs, INCLUDE / "benchsp_compat.hpp", INCLUDE / "bsp.h", LIB]
    if not force and COMPAT_LIB.exists() and COMPAT_LIB.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return COMPAT_LIB
    tmp = COMPAT_LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", f"-I{INCLUDE}", f"-I{CUDA_HOME}/include",
           "-o", str(tmp), *map(str, srcs), f"-L{LIB.parent}", "-lbspmv", f"-L{CUDA_HOME}/lib64", "-lcusparse",
           "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{CUDA_HOME}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compat link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, COMPAT_LIB)
    return COMPAT_LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True))


if __name__ == "__main__":
    main()
