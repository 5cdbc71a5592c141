"""Build recipe of the in-tree shared libraries ``nlos_lbm/liblbm_b200.so``
(the product) and ``nlos_lbm/liblbm_b200_check.so`` (the same sources with
-DLBM_CHECK: device accesses tested against their arrays' extents; loaded
instead of the product when NLOS_LBM_CHECK=1).

kernels.cu is compiled by nvcc for sm_100a only; the host C++ (api.cpp,
geometry.cpp) by g++ with -ffp-contract=off so its FP64 arithmetic matches the
reference's rounding.  The CUDA runtime is linked statically, so the library
needs only the NVIDIA driver at run time.  Run ``python -m nlos_lbm.build`` or call
``build()``.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)                      # city-scale-nlos-acoustic-engine-code_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "liblbm_b200.so")
BUILD_CHECK = os.path.join(ROOT, "_build_check")
LIB_CHECK = os.path.join(PKG, "liblbm_b200_check.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["kernels.cu", "adjoint.cu", "scheme_a.cu", "voxel.cu"]
# voxel.cu must round every FP64 expression as the host does (no FMA contraction)
CU_FLAGS = {"voxel.cu": ["-fmad=false"]}
CXX_SOURCES = ["api.cpp", "geometry.cpp"]
HEADERS = ["adjoint.hpp", "check.cuh", "device.hpp", "geometry.hpp", "lattice.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)
    return r.stdout + r.stderr


def build(verbose=False, force=False, ptxas_verbose=False, check=False):
    """Compile the library if any source is newer than it; returns its path.
    check: the bounds-checked library instead of the product."""
    build_dir, lib = (BUILD_CHECK, LIB_CHECK) if check else (BUILD, LIB)
    defs = ["-DLBM_CHECK"] if check else []
    os.makedirs(build_dir, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "nlos_lbm.h")]
    objs = []
    log = ""
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(build_dir, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-ccbin", CXX, "-Xcompiler", "-fPIC",
                   "-I" + INCLUDE, "-I" + CSRC, *defs, *CU_FLAGS.get(src, []), "-c", s, "-o", o]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
            log += _run(cmd, verbose)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(build_dir, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
                   "-Wall", "-Wno-unknown-pragmas", *defs, "-I" + INCLUDE, "-I" + CSRC,
                   "-I" + os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o]
            log += _run(cmd, verbose)
    if force or _newer(lib, objs):
        tmp = lib + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-ccbin", CXX, "-Xcompiler", "-fopenmp", "-o", tmp, *objs, "-lgomp"]
        log += _run(cmd, verbose)
        shutil.move(tmp, lib)
    return lib if not ptxas_verbose else (lib, log)


if __name__ == "__main__":
    res = build(verbose=True, force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv,
                check="--check" in sys.argv)
    print(res if isinstance(res, str) else res[1])
