"""In-tree build of the native parts (no JIT cache, so the built files travel with the tree).

    python -m allen_b200.build            # chain (nvcc, sm_100a) + generator and MDF input (g++)

The CUDA library is compiled for sm_100a only, with -fmad=false: the cluster
positions, phi values and track fits must round exactly like the reference's
CPU build, which never fuses a multiply with an add.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "_lib")
INCLUDE = os.path.join(REPO, "include")


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xptxas", "-v", "--expt-relaxed-constexpr",
]


def build_chain(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    target = os.path.join(LIB_DIR, "libvelo_b200.so")
    cus = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = cus + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    if not force and not _stale(target, deps):
        return target
    objs = [os.path.join(LIB_DIR, os.path.basename(cu) + ".o") for cu in cus]

    def compile_one(cu, obj):
        cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", cu, "-o", obj]
        return cu, subprocess.run(cmd, capture_output=True, text=True)

    # one nvcc per translation unit, in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cus), os.cpu_count() or 1)) as pool:
        for cu, r in pool.map(lambda a: compile_one(*a), zip(cus, objs)):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {cu}:\n{r.stderr}")
            if verbose:
                sys.stderr.write(r.stderr)
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", target, *objs,
           "-lcudart", "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    for o in objs:
        os.remove(o)
    return target


def build_generator(force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    target = os.path.join(LIB_DIR, "libvelo_gen.so")
    src = os.path.join(CSRC, "velo_generator.cpp")
    if not force and not _stale(target, [src, os.path.join(INCLUDE, "velo_generator.h")]):
        return target
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-I", INCLUDE, "-o", target, src]
    subprocess.run(cmd, check=True)
    return target


def build_io(force: bool = False) -> str:
    """Host-only MDF index and VELO transpose (include/velo_io.h); no CUDA dependency."""
    os.makedirs(LIB_DIR, exist_ok=True)
    target = os.path.join(LIB_DIR, "libvelo_io.so")
    src = os.path.join(CSRC, "velo_io.cpp")
    if not force and not _stale(target, [src, os.path.join(INCLUDE, "velo_io.h")]):
        return target
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-Wall", "-I", INCLUDE, "-o", target, src]
    subprocess.run(cmd, check=True)
    return target


def main():
    build_generator(force="--force" in sys.argv)
    build_io(force="--force" in sys.argv)
    build_chain(force="--force" in sys.argv, verbose="-v" in sys.argv)


if __name__ == "__main__":
    main()
