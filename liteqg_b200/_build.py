"""Builds the package's native library in-tree.

``liteqg_b200/_lib/liblqg.so`` is the C-ABI library declared in
``include/lqg.h``: every ``csrc/*.cu`` file compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), objects under ``_build/``,
linked with the static CUDA runtime. Rebuilds only what changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "liblqg.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2", "-ccbin", "/usr/bin/g++",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + [
        os.path.join(ROOT, "include", "lqg.h")
    ]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, jobs: int | None = None) -> str:
    """Compiles and links liblqg.so if any source changed; returns its path."""
    nvcc = _nvcc()
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = _headers()
    jobs_list = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            cmd = [nvcc, *ARCH, *NVFLAGS, "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o]
            jobs_list.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return cmd

    if jobs_list:
        n = jobs or min(len(jobs_list), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(n) as ex:
            list(ex.map(run, jobs_list))
    if jobs_list or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs,
             "-Xlinker", "--exclude-libs,ALL"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
