"""Builds the in-tree CUDA library ``libmeikey_b200.so`` for sm_100a with nvcc.

The library holds the kernels (csrc/kernels.cu) and the C ABI (csrc/api.cpp,
csrc/host25519.cpp, ...); it links the CUDA runtime statically so that the .so only
needs the driver at run time.  Every source is compiled to its own object in parallel
(objects in csrc/_build/, rebuilt when their source or any header changed), then linked.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libmeikey_b200.so")
SOURCES = ["kernels.cu", "dfa_build.cu", "api.cpp", "host25519.cpp", "regex.cpp", "tune.cpp", "serve.cpp",
           "keyfile.cpp"]
HEADERS = ["fe32.cuh", "fe26.cuh", "fe51.cuh", "ge.cuh", "hash.cuh", "kernels.h", "types.h", "host25519.h", "hitsort.h",
           "abi_guard.h", "jobs.h", "regex.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-fvisibility=hidden"]
LINK_FLAGS = ARCH + ["-shared", "-cudart", "static"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _headers_mtime():
    deps = [os.path.join(CSRC, f) for f in HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "meikey_b200.h"))
    deps.append(__file__)
    return max(os.path.getmtime(d) for d in deps if os.path.exists(d))


def _obj(src):
    return os.path.join(OBJ, src + ".o")


def _stale_objects(force):
    hdr = _headers_mtime()
    out = []
    for src in SOURCES:
        o = _obj(src)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(hdr, os.path.getmtime(os.path.join(CSRC, src))):
            out.append(src)
    return out


def _stale_lib():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(not os.path.exists(_obj(s)) or os.path.getmtime(_obj(s)) > t for s in SOURCES)


def build(force=False, verbose=False):
    """Compile the library if a source is newer than it; returns its path."""
    todo = _stale_objects(force)
    if not todo and not _stale_lib():
        return LIB
    os.makedirs(OBJ, exist_ok=True)

    def compile_one(src):
        cmd = [_nvcc(), *COMPILE_FLAGS, "-c", os.path.join(CSRC, src), "-o", _obj(src) + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, cwd=CSRC)
        os.replace(_obj(src) + ".tmp", _obj(src))

    with ThreadPoolExecutor(max(1, len(todo))) as ex:
        list(ex.map(compile_one, todo))
    cmd = [_nvcc(), *LINK_FLAGS, "-o", LIB + ".tmp"] + [_obj(s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
