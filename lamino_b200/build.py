"""Build the lamino_b200 CUDA library in-tree (sm_100a).

    python -m lamino_b200.build            # -> lamino_b200/liblamino_b200.so

nvcc cross-compiles for sm_100a without a GPU.  cudart is linked statically;
cuFFT is linked dynamically from the CUDA toolkit (rpath to its lib64).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblamino_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(HERE, "..", "include", "lamino.h")]
    return any(os.path.getmtime(f) > t for f in deps if os.path.exists(f))


def build(verbose: bool = False, force: bool = False, ptxas_v: bool = False) -> str:
    """Compile each .cu into an object in parallel (lamino_b200/_build/), then link
    the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    nvcc = nvcc_path()
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "lib64")
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3"]
    if ptxas_v:
        flags = ["-Xptxas", "-v", *flags]

    def compile_one(src):
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [nvcc, *flags, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        return src, obj, r

    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, srcs))
    for src, _, r in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
        if verbose or ptxas_v:
            sys.stderr.write(r.stderr)
    cmd = [nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *[o for _, o, _ in results],
           f"-L{cuda_lib}", "-lcufft", "-Xlinker", f"-rpath={cuda_lib}"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link of liblamino_b200.so failed")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_v="--ptxas-v" in sys.argv)
    print(LIB)
