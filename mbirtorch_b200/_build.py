"""Build recipe for the sm_100a shared library ``libmbir_b200.so``.

The library is compiled IN-TREE with nvcc (no torch headers: the C ABI takes
plain pointers), so the built file travels with the source tree.  Run
``python -m mbirtorch_b200._build`` or call :func:`build`.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB_NAME = "libmbir_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)
SOURCES = ["capi.cu"]
HEADERS = ["mbir_common.cuh", "projectors.cuh", "vcd.cuh", "batch.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put CUDA's bin on PATH")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "mbir_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date():
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force=False, verbose=False, extra_flags=()):
    """Compile csrc/*.cu for sm_100a into mbirtorch_b200/libmbir_b200.so."""
    if not force and up_to_date():
        return LIB_PATH
    tmp = LIB_PATH + ".tmp%d" % os.getpid()
    cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared",
           "-Xcompiler", "-fPIC", "-I", INCLUDE, "-o", tmp,
           *[os.path.join(CSRC, s) for s in SOURCES], *extra_flags]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
