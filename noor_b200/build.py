"""Builds libnoor_b200.so in-tree for sm_100a.

CUDA sources are compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a``
(no fast-math: the sky and BSDF routines use CUDA's accurate libm), host C++
sources by g++ with ``-ffp-contract=off`` so the scene builder's float results
do not depend on contraction.  The shared library links the CUDA runtime
statically and exports the C-ABI of include/noor_b200.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libnoor_b200.so"
OBJ = ROOT / "_build" / "noor_b200"

CU_SOURCES = ["kernels.cu", "envmap.cu", "context.cu", "wavefront.cu", "adjoint.cu", "noalloc.cu", "tonemap.cu",
              "bvh_gpu.cu"]
# the GPU BVH builder rounds its split search as the host builder does
CU_EXTRA = {"bvh_gpu.cu": ["-fmad=false"]}
CPP_SOURCES = ["scene_build.cpp", "wide_bvh.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-std=c++17", "-O3", "-lineinfo",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xptxas", "-warn-spills",
]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-pthread", "-ffp-contract=off", "-fvisibility=hidden", "-Wall"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, out: Path = OUT, obj: Path = OBJ,
          defines: tuple = ()) -> Path:
    """Compile every source that changed and relink the library (into `out`,
    objects under `obj`, with extra -D `defines`)."""
    OBJ_, OUT_ = obj, out
    obj.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "noor_b200.h"]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = OBJ_ / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([nvcc, *NVCC_FLAGS, *CU_EXTRA.get(src, []), *[f"-D{d}" for d in defines], "-c", str(s),
                         "-o", str(o)])
    for src in CPP_SOURCES:
        s = CSRC / src
        o = OBJ_ / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++", *CXX_FLAGS, "-I", str(ROOT / "include"), "-c", str(s), "-o", str(o)])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or _stale(OUT_, objs):
        tmp = OUT_.with_suffix(".so.tmp")
        _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
              *[str(o) for o in objs], "-o", str(tmp)])
        os.replace(tmp, OUT_)
    if verbose:
        print(f"built {OUT_}")
    return OUT_


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
