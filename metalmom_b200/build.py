"""Build libmetalmom.so (CUDA kernels + C ABI) for sm_100a, in tree.

    python metalmom_b200/build.py [--force]

(run as a script: importing the package itself needs the built library).

Sources: metalmom_b200/csrc/*.cu; output: metalmom_b200/_lib/libmetalmom.so.
The CUDA runtime is linked statically, so the library needs only the driver.
"""

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libmetalmom.so")
SOURCES = ["frontend_kernels.cu", "frontend_warp.cu", "runtime.cu", "abi.cu", "noalloc.cu", "server.cu", "plan.cu", "dft_gemm.cu", "features.cu", "istft.cu", "spec_ops.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "-DMM_BUILDING_LIBRARY", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "metalmom.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src):
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [NVCC] + ARCH + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    subprocess.check_call(cmd)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _deps() + [os.path.abspath(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(len(SOURCES)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
    subprocess.check_call(cmd)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
