"""Build libluminis_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python luminis-mc_b200/build.py [--force] [--verbose]

Output: luminis-mc_b200/luminis_mc_b200/lib/libluminis_b200.so.  The CUDA
runtime is linked statically, so the library depends only on the driver.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")
OUT_DIR = os.path.join(HERE, "luminis_mc_b200", "lib")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libluminis_b200.so")
CHECKED_LIB = os.path.join(OUT_DIR, "libluminis_b200_checked.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Binary32 division and square root by the fast approximations, binary32 denormals
# flushed: the FP32 transport's results stay within its parity tolerances and the sweep,
# mixture and absorption kernels run 6-12 % faster.  Binary64 arithmetic is unaffected
# (the Mie tables in lmc_tables.cu use explicitly rounded binary64 operations).
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-prec-div=false", "-prec-sqrt=false", "-ftz=true",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False,
          bounds_check: bool = False) -> str:
    """Build the library (bounds_check: the debug variant libluminis_b200_checked.so, whose
    kernels check every table and tally index and report failed sites)."""
    obj_dir = OBJ_DIR + ("_checked" if bounds_check else "")
    lib = CHECKED_LIB if bounds_check else LIB
    defines = ["-DLMC_BOUNDS_CHECK"] if bounds_check else []
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(obj_dir, exist_ok=True)
    cu, cpp = _sources()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "luminis_b200.h"))
    objs = []

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or ptxas_info:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")

    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(obj_dir, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            run([nvcc(), *ARCH, *NVCC_FLAGS, *defines, *extra, "-c", src, "-o", obj])
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")   # NVTX headers
    for f in cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(obj_dir, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            run(["g++", *CXX_FLAGS, f"-I{cuda_inc}", "-c", src, "-o", obj])
    if force or _stale(lib, objs):
        run([nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-lpthread"])
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--bounds-check", action="store_true",
                    help="the debug variant libluminis_b200_checked.so")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_info, a.bounds_check))
