"""Builds the native library and command-line drivers in-tree for sm_100a.

    python -m geneva_b200.build            # geneva_b200/lib/{libgeneva.so,gpumine,gpumineSV}

The library is plain CUDA C++ behind a C ABI (include/geneva.h); nothing here
depends on torch.  Objects are rebuilt only when a source or header is newer.
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
LIB = PKG / "lib"
OBJ = LIB / "obj"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-sign-compare", f"-I{ROOT / 'include'}"]

CU_SOURCES = ["gva_engine.cu", "gva_batch.cu", "gva_static.cu", "gva_mni.cu", "gva_dplan.cu"]
CPP_SOURCES = ["gva_plan.cpp", "gva_graph.cpp", "gva_capi.cpp", "gva_mine.cpp", "gva_convert.cpp", "gva_text.cpp",
               "gva_pool.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home() -> Path:
    return Path(nvcc()).resolve().parent.parent


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r


def build(verbose: bool = False) -> Path:
    """Compile everything; returns the path of libgeneva.so."""
    LIB.mkdir(parents=True, exist_ok=True)
    OBJ.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.inc")) + [ROOT / "include" / "geneva.h"]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        o = OBJ / (src + ".o")
        objs.append(o)
        if _newer(o, [CSRC / src, *headers]):
            jobs.append([nvcc(), *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(o)])
    cxx = shutil.which("g++") or "g++"  # system g++: shared libstdc++ (see oracle/Makefile)
    inc = f"-I{cuda_home() / 'include'}"
    for src in CPP_SOURCES + ["gva_cli.cpp"]:
        if src == "gva_cli.cpp":
            continue
        o = OBJ / (src + ".o")
        objs.append(o)
        if _newer(o, [CSRC / src, *headers]):
            jobs.append([cxx, *CXX_FLAGS, inc, "-c", str(CSRC / src), "-o", str(o)])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for r in ex.map(_run, jobs):
            if verbose and r.stderr:
                print(r.stderr, file=sys.stderr)
    so = LIB / "libgeneva.so"
    if _newer(so, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", str(so), *map(str, objs), "-Xlinker", "-soname=libgeneva.so",
              "-lstdc++"])
    conv = LIB / "gvaconvert"
    if _newer(conv, [so, CSRC / "gva_convert_main.cpp", ROOT / "include" / "geneva.h"]):
        _run([cxx, *CXX_FLAGS, str(CSRC / "gva_convert_main.cpp"), "-o", str(conv), f"-L{LIB}", "-lgeneva",
              "-Wl,-rpath,$ORIGIN", "-lstdc++"])
    for name, mode in (("gpumine", 0), ("gpumineSV", 1)):
        exe = LIB / name
        if _newer(exe, [so, CSRC / "gva_cli.cpp", ROOT / "include" / "geneva.h"]):
            _run([cxx, *CXX_FLAGS, f"-DGVA_CLI_MODE={mode}", str(CSRC / "gva_cli.cpp"), "-o", str(exe),
                  f"-L{LIB}", "-lgeneva", "-Wl,-rpath,$ORIGIN", "-lstdc++"])
    return so


if __name__ == "__main__":
    print(build(verbose=True))
