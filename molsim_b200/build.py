"""Build recipe for the B200 library (libmolsim_gpu.so, in-tree).

    python -m molsim_b200.build          # builds molsim_b200/libmolsim_gpu.so

Compiles every CUDA source for sm_100a with nvcc (cross-compiles without a GPU).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIB = os.path.join(HERE, "libmolsim_gpu.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("engine.cu", "noalloc.cu", "polyatomic.cu", "setup.cpp")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + \
    [os.path.join(ROOT, "include", "molsim_gpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-shared", "-cudart", "static",
]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS if os.path.exists(p))


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    nvcc = os.path.join(CUDA, "bin", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + list(extra) + ["-I", os.path.join(ROOT, "include"), "-o", LIB] + SOURCES + [
        "-L", os.path.join(CUDA, "lib64"), "-lcufft", "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
