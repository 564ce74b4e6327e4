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
    build_pyelsa(force)
    return LIB


def build_pyelsa(force=False):
    """The pybind11 module elsa_b200._pyelsa (csrc/pyelsa_ext.cpp over include/elsa_b200.hpp),
    linked against libelsa_b200.so beside it. Skipped when pybind11 is not installed."""
    try:
        import pybind11
    except ImportError:
        return None
    import sysconfig
    src = os.path.join(CSRC, "pyelsa_ext.cpp")
    out = os.path.join(HERE, "_pyelsa" + sysconfig.get_config_var("EXT_SUFFIX"))
    deps = [src, LIB, os.path.join(ROOT, "include", "elsa_b200.hpp"),
            os.path.join(ROOT, "include", "elsa_b200.h")]
    if not force and not _stale(out, deps):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
           "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", src,
           "-o", out, "-L" + HERE, "-lelsa_b200", "-Wl,-rpath,$ORIGIN",
           "-L/usr/local/cuda/lib64", "-lcudart"]
    _compile(cmd)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
