"""Build helper for the C++-layer example (tests/cpp/cxx_layer_example.cpp)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(out_dir):
    exe = os.path.join(out_dir, "cxx_layer_example")
    lib_dir = os.path.join(ROOT, "elsa_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-o", exe,
           os.path.join(HERE, "cpp", "cxx_layer_example.cpp"),
           "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
           "-L" + lib_dir, "-lelsa_b200", "-Wl,-rpath," + lib_dir,
           "-L/usr/local/cuda/lib64", "-lcudart"]
    subprocess.check_call(cmd)
    return exe
