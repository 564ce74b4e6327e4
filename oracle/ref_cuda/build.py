"""Build recipe for oracle/_ref/librefcuda.so: elsa's own CUDA projector kernels
(projectors_cuda/projector_kernels/TraverseJosephsCUDA.cu, TraverseSiddonsCUDA.cu,
ProjectVoxelsCUDA.cu), compiled from the reference sources where they lie, with the stand-in
headers in shim/ and the host harness refcuda.cu. TEST INFRASTRUCTURE ONLY: the library lets the
GPU tests time the reference's kernels beside this library's on the same device.

Run where the reference tree exists: ELSA_REFERENCE_DIR=<root of the reference checkout>
python -m oracle.ref_cuda.build (the recipe looks for <root>/elsa/projectors_cuda/...; without the
variable it looks at the checkout location of the build container). The built library travels
with the repository snapshot; the reference tree is not needed to load it."""
import os
import subprocess
import sys

# root of the reference checkout (its elsa/ source tree), for this build recipe only
REFERENCE = os.path.join(os.environ.get("ELSA_REFERENCE_DIR", "/root/reference"), "elsa")
_HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(os.path.dirname(_HERE), "_ref")
LIB = os.path.join(OUT_DIR, "librefcuda.so")
KERNELS = ["TraverseJosephsCUDA.cu", "TraverseSiddonsCUDA.cu", "ProjectVoxelsCUDA.cu"]


def available():
    return os.path.isdir(os.path.join(REFERENCE, "projectors_cuda", "projector_kernels"))


def build(force=False):
    """Compile the library; returns its path, or None when the reference tree is absent."""
    if not available():
        return None
    kdir = os.path.join(REFERENCE, "projectors_cuda", "projector_kernels")
    srcs = [os.path.join(_HERE, "refcuda.cu")] + [os.path.join(kdir, k) for k in KERNELS]
    deps = srcs + [os.path.join(_HERE, "shim", f) for f in os.listdir(os.path.join(_HERE, "shim"))]
    if (not force and os.path.exists(LIB)
            and all(os.path.getmtime(LIB) >= os.path.getmtime(f) for f in deps)):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
           "-shared", "-Xcompiler", "-fPIC", "-Wno-deprecated-gpu-targets",
           "-I" + os.path.join(_HERE, "shim"), "-I" + kdir,
           "-I" + os.path.join(REFERENCE, "projectors"),
           "-I" + os.path.join(REFERENCE, "core", "Utilities"),
           "-o", LIB] + srcs
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    path = build(force="--force" in sys.argv)
    print(path or "reference tree not present: nothing built")
