"""Build libdmrgb200.so in-tree (sm_100a device code + host schedule builder).

Usage: python maquis-dmrg_b200/build.py [--force]
The library lands in maquis-dmrg_b200/dmrgb200/libdmrgb200.so so that it
travels with the source tree; object files go to maquis-dmrg_b200/_build/.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
OUT = HERE / "dmrgb200" / "libdmrgb200.so"
INCLUDE = HERE.parent / "include"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))

CXX_SOURCES = ["coupling.cpp", "schedule.cpp", "plan.cpp", "capi.cpp", "per_block.cpp"]
CU_SOURCES = ["kernels_fp64.cu", "noalloc.cu", "jd.cu", "jd_graph.cu", "ozaki.cu", "adjoint.cu", "block_svd.cu",
              "alpha_dm.cu"]
HEADERS = ["symm.hpp", "mpo.hpp", "coupling.hpp", "boundary_index.hpp", "schedule.hpp", "plan.hpp",
           "device.hpp", "async_copy.cuh"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function"]


def _run(cmd: list[str], log: Path | None = None) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.write_text(res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [INCLUDE / "dmrgb200.h"]
    objs = []
    for src in CXX_SOURCES:
        obj = BUILD / (src + ".o")
        if force or _stale(obj, [CSRC / src] + hdrs):
            _run(["g++", *CXX_FLAGS, f"-I{CUDA}/include", f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(obj)])
        objs.append(obj)
    for src in CU_SOURCES:
        obj = BUILD / (src + ".o")
        if force or _stale(obj, [CSRC / src] + hdrs):
            _run([str(CUDA / "bin" / "nvcc"), *NVCC_FLAGS, f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(obj)],
                 log=BUILD / (src + ".ptxas.txt"))
        objs.append(obj)
    if force or _stale(OUT, objs):
        _run(["g++", "-shared", "-o", str(OUT), *map(str, objs), f"-L{CUDA}/lib64", "-lcudart", "-lcublas", "-fopenmp",
              f"-Wl,-rpath,{CUDA}/lib64"])
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
