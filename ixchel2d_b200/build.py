"""Build libixb.so in-tree for sm_100a with nvcc.

Run ``python -m ixchel2d_b200.build`` (or call :func:`build`).  Objects go to
``ixchel2d_b200/_build/``; the shared library to ``ixchel2d_b200/libixb.so``
and the case driver (PROGRAM IXCHEL2D on the library) to
``ixchel2d_b200/ixchel2d_gpu``.
Rebuilds only what changed (any header change rebuilds every object).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libixb.so"
DRIVER = PKG / "ixchel2d_gpu"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the coefficient assembly is bit-identical to the reference's
# IEEE evaluation only without FMA contraction; kernels that want FMAs
# request them explicitly.
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "-I", str(INCLUDE)]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-I", str(INCLUDE)]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build libixb.so")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(src: Path, obj: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return t < src.stat().st_mtime or t < newest_header


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    if src.suffix == ".cu":
        flags = list(NVFLAGS)
        if src.stem.endswith(("_fast", "_mixed")):
            # the fast and mixed-precision (tolerance-checked) kernels may
            # contract a*b+c into FMA
            flags[flags.index("-fmad=false")] = "-fmad=true"
        cmd = [_nvcc(), *ARCH, *flags, *extra, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [HOST_CXX, *CXXFLAGS, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, ptxas_v: bool = False) -> Path:
    """Compile every CUDA/C++ source of the package and link libixb.so."""
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    extra = ["-Xptxas", "-v"] if ptxas_v else []
    jobs = []
    objs = []
    for s in srcs:
        o = BUILD / (s.name + ".o")
        objs.append(o)
        if ptxas_v or _stale(s, o, newest_header):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for obj, log in ex.map(lambda j: _compile(j[0], j[1], extra), jobs):
                if verbose or ptxas_v:
                    print(f"[ixb build] {obj.name}\n{log}", file=sys.stderr)
    for stale in BUILD.glob("*.o"):
        if stale not in objs:
            stale.unlink()
    newest_obj = max(o.stat().st_mtime for o in objs)
    if jobs or not LIB.exists() or LIB.stat().st_mtime < newest_obj:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-ldl",
               "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_driver()
    return LIB


def build_driver() -> Path:
    """Link the ixchel2d_gpu case driver against libixb.so (found next to it
    at run time through an $ORIGIN rpath)."""
    srcs = [CSRC / "driver" / "ixchel2d_gpu.cpp", CSRC / "ixb_listdir.cpp"]
    deps = srcs + [LIB, CSRC / "ixb_listdir.h", INCLUDE / "ixb.h"]
    if DRIVER.exists() and DRIVER.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return DRIVER
    tmp = DRIVER.with_name(DRIVER.name + ".tmp")
    cmd = [HOST_CXX, *CXXFLAGS, "-pthread", "-o", str(tmp), *map(str, srcs), "-L", str(PKG), "-lixb",
           "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, DRIVER)
    return DRIVER


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv)
    print(LIB)
