"""Build recipe for the C oracle / CPU baseline (test infrastructure).

Compiles ``oracle/refcpu.c`` into ``oracle/_build/librefcpu.so`` with plain
gcc.  MetalMom itself (Swift + Apple Accelerate) cannot be compiled on Linux,
so there is no ``oracle/_ref`` build of the reference.
"""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "librefcpu.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "refcpu.c")
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(src)):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-std=c11",
           "-D_GNU_SOURCE", "-Wall", "-o", LIB, src, "-lm", "-lpthread"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
