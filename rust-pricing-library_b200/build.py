"""Build recipe of the engine library (libmcg.so) for sm_100a.

Every translation unit is compiled by nvcc for `-gencode arch=compute_100a,code=sm_100a`.
FP64 units use -fmad=false so a*b+c rounds twice, like the reference's Rust
arithmetic; the objects are linked into one shared library in the package
directory, next to the Python host that loads it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "rust_pricing_b200")
LIB = os.path.join(OUT_DIR, "libmcg.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills"]
# (source, extra flags)
UNITS = [
    ("mcg_lv.cu", ["-fmad=false"]),
    ("mcg_lv_adjoint.cu", ["-fmad=false"]),
    ("mcg_bs.cu", ["-fmad=false"]),
    ("mcg_bs_risk.cu", ["-fmad=false"]),
    ("mcg_dual.cu", ["-fmad=false"]),
    ("mcg_setup.cu", ["-fmad=false"]),
    ("mcg_host.cu", ["-fmad=false"]),
    ("mcg_noalloc.cu", ["-fmad=false"]),
    ("mcg_lsm.cu", ["-fmad=false"]),
    ("mcg_mlp.cu", []),
    ("mcg_book.cu", ["-fmad=false"]),
    ("mcg_lv32.cu", []),
    ("mcg_vegakt.cu", []),
    ("mcg_multi.cu", ["-fmad=false"]),
    ("mcg_bump.cu", ["-fmad=false"]),
]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "mcg.h"))
    return hs


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objects = []
    jobs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objects.append(o)
        if force or _stale(o, [s, *headers, __file__]):
            cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", s, "-o", o]
            jobs.append(cmd)
    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)
        return r
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as pool:
        list(pool.map(run, jobs))
    if force or jobs or _stale(LIB, objects):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objects, "-lcudart"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
