"""Build libfftlib_b200.so in-tree with nvcc for sm_100a.

    python -m c7x_fftlib_b200._build [--force] [-j N]

Every .cu under csrc/ is compiled to an object in _build/ (in parallel,
skipped when up to date) and linked into c7x_fftlib_b200/libfftlib_b200.so
with the CUDA runtime linked statically.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libfftlib_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-I", CSRC, "-I", os.path.join(INC, "fftlib_b200"), "-I", INC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INC, "**", "*.h"), recursive=True)


def _compile(src: str, force: bool, hdr_mtime: float) -> tuple[str, float]:
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
        return obj, 0.0
    import time
    t = time.time()
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, time.time() - t


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    # the widest engine instantiation compiles longest: start it first
    srcs.sort(key=lambda s: 0 if "e32" in s else 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hdr_mtime), srcs))
    if verbose:
        for (o, t) in objs:
            if t:
                print(f"  compiled {os.path.basename(o)} in {t:.1f}s")
    newest = max(os.path.getmtime(o) for o, _ in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *[o for o, _ in objs], "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    print(build(a.force, a.j, verbose=True))
    sys.exit(0)
