"""Build `libtpagmg.so` in-tree for sm_100a (B200).

Host set-up sources are compiled by g++, device sources by nvcc with
`-gencode arch=compute_100a,code=sm_100a`; the shared library lands in
`tpagmg/_lib/` next to the Python host mirror so that it travels with the
source tree.  Rebuilds only what changed.
"""
import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "tpagmg" / "_lib"
BUILD = HERE / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_SRC = ["mesh.cpp", "metric.cpp", "hierarchy.cpp", "structure.cpp", "tiles.cpp", "cmdgfm.cpp"]
DEVICE_SRC = ["device.cu", "solve_fused.cu", "solve_fast.cu", "noalloc.cu", "adjoint.cu", "batch.cu", "autotune.cu", "refresh.cu", "projection.cu", "cmdgfm.cu", "api.cpp"]


def _stale(target, deps):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose=False):
    OUT.mkdir(parents=True, exist_ok=True)
    BUILD.mkdir(parents=True, exist_ok=True)
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "tpagmg.h"]
    objs = []
    for src in HOST_SRC:
        obj = BUILD / (src + ".o")
        if _stale(obj, [CSRC / src] + headers):
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function",
                   "-I/usr/local/cuda/include", "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(obj)
    for src in DEVICE_SRC:
        obj = BUILD / (src + ".o")
        if _stale(obj, [CSRC / src] + headers):
            cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
                   "--expt-relaxed-constexpr", "-x", "cu", "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        objs.append(obj)
    lib = OUT / "libtpagmg.so"
    if _stale(lib, objs):
        cmd = [NVCC, "-shared", *ARCH, "-o", str(lib), *map(str, objs), "-Xcompiler", "-fopenmp", "-lgomp"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
