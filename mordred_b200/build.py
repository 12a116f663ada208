"""Build the in-tree CUDA library ``mordred_b200/libmordred_b200.so`` for sm_100a.

The library holds every kernel and the C ABI declared in ``include/mordred_b200.h``.
It is compiled with nvcc directly (no JIT cache), so the built file travels with the
source tree. Run ``python -m mordred_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmordred_b200.so")

SOURCES = ["capi.cu", "star.cu", "star_special.cu", "star_wide.cu", "build.cu", "listq.cu", "noalloc.cu", "batch.cu", "compact.cu", "mlp.cu", "cpu_engine.cpp",
           "segcache.cpp", "costmodel.cpp"]
# host code: portable x86-64 with AVX2 (the library is built on one machine and run on another)
HOST_FLAGS = ["-O3", "-march=x86-64-v3", "-std=c++17", "-fPIC", "-pthread"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_INCLUDE = "/usr/local/cuda/include"


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return "nvcc"


def _sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES]


def _deps() -> list[str]:
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for base, _, files in os.walk(d):
            out += [os.path.join(base, f) for f in files if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    return res.stderr


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile the library if any source is newer than it; return its path.

    Each translation unit is compiled to an object in parallel, then linked."""
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc(), *GENCODE, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-O3", "-I", os.path.join(ROOT, "include")]
    if ptxas_verbose:
        common += ["-Xptxas", "-v"]
    jobs = []
    for src in _sources():
        stem, ext = os.path.splitext(os.path.basename(src))
        obj = os.path.join(objdir, stem + ".o")
        if ext == ".cpp":
            jobs.append((["g++", *HOST_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CUDA_INCLUDE, "-c", "-o",
                          obj, src], obj))
        else:
            jobs.append(([*common, "-c", "-o", obj, src], obj))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(lambda j: _run(j[0], verbose), jobs))
    if ptxas_verbose:
        print("\n".join(logs), file=sys.stderr)
    _run([nvcc(), *GENCODE, "--shared", "-o", LIB + ".tmp", *[o for _, o in jobs], "-lpthread"], verbose)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="-v" in sys.argv)
    print(LIB)
