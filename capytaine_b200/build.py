"""Build the sm_100a shared library ``capytaine_b200/libcapytaine_b200.so``.

Each ``csrc/*.cu`` is compiled by nvcc for ``compute_100a``/``sm_100a`` and the
objects are linked into one shared library with the CUDA runtime linked
statically (the library then works next to any other CUDA runtime in the
process, e.g. torch's).  Objects are rebuilt only when a source or header is
newer.  Usage: ``python -m capytaine_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcapytaine_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
# Files that must not contract multiply-adds (float32 rational approximations
# restated operation by operation).
NO_FMA = {"tabulation.cu"}


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cutlass_include():
    try:
        import flashinfer  # noqa: F401  (header tree only)
        d = os.path.join(os.path.dirname(flashinfer.__file__), "data", "cutlass", "include")
    except Exception:
        d = ""
    if d and os.path.isdir(d):
        return ["-I", d]
    return []


def _needs(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    extra = _cutlass_include()
    jobs = []
    objs = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _needs(obj, [src] + headers):
            flags = list(COMMON) + extra
            if os.path.basename(src) in NO_FMA:
                flags.append("-fmad=false")
            jobs.append([nvcc, *ARCH, *flags, "-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed for {cmd[-3]}:\n{p.stdout}\n{p.stderr}")
        if verbose and (p.stdout or p.stderr):
            print(p.stdout, p.stderr)

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not os.path.exists(LIB):
        link = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        run(link)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
