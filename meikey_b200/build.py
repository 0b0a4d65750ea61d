"""Builds the in-tree CUDA library ``libmeikey_b200.so`` for sm_100a with nvcc.

The library holds the kernels (csrc/kernels.cu) and the C ABI (csrc/api.cpp,
csrc/host25519.cpp); it links the CUDA runtime statically so that the .so only
needs the driver at run time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmeikey_b200.so")
SOURCES = ["kernels.cu", "api.cpp", "host25519.cpp", "regex.cpp", "tune.cpp", "serve.cpp", "keyfile.cpp"]
HEADERS = ["fe32.cuh", "fe26.cuh", "fe51.cuh", "ge.cuh", "hash.cuh", "kernels.h", "types.h", "host25519.h", "hitsort.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden",
    "-shared", "-cudart", "static",
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "meikey_b200.h"))
    deps.append(__file__)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library if a source is newer than it; returns its path."""
    if not force and not _stale():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", LIB + ".tmp"] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
