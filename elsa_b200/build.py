"""Build the elsa_b200 native library (libelsa_b200.so) in-tree with nvcc for sm_100a.

Usage: python -m elsa_b200.build [--force]

Every translation unit is compiled for sm_100a only. raysetup.cu is compiled with --fmad=false
(its float arithmetic must round exactly like the reference's CPU path); host geometry is compiled
with -ffp-contract=off for the same reason.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libelsa_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler",
              "-ffp-contract=off", "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall",
             "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include"]

# Extra nvcc flags for experiments (e.g. -DELSA_ADJ_NW=2); empty for the product build.
CUDA_FLAGS += os.environ.get("ELSA_B200_NVCC_EXTRA", "").split()

# (source, extra flags)
CUDA_UNITS = [
    ("raysetup.cu", ["--fmad=false"]),
    ("joseph.cu", []),
    ("joseph_tma.cu", []),
    ("siddon.cu", []),
    ("voxel.cu", ["--fmad=false"]),
    ("vecops.cu", []),
    ("noalloc.cu", []),
    ("lutproj.cu", []),
    ("solvers.cu", []),
]
CXX_UNITS = [
    ("geometry.cpp", []),
    ("luts.cpp", []),
    ("capi.cpp", []),
    ("tune.cpp", []),
    ("io.cpp", []),
]
HEADERS = ["internal.cuh", "raysetup.cuh", "joseph_tma.cuh", "projector.hpp", "geometry.hpp", "vecops.cuh",
           "solvers.hpp", "luts.hpp", "voxel.hpp", "tune.hpp", "io.hpp"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include",
                                                                        "elsa_b200.h")]
    jobs = []
    objs = []
    for src, extra in CUDA_UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([NVCC] + ARCH + CUDA_FLAGS + extra + ["-c", s, "-o", o])
    for src, extra in CXX_UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++"] + CXX_FLAGS + extra + ["-c", s, "-o", o])
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for err in ex.map(_compile, jobs):
            if verbose and err:
                sys.stderr.write(err)
    if force or jobs or _stale(LIB, objs):
        _compile([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
