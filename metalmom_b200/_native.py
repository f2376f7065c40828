"""cffi loader for libmetalmom.so (ABI mode, as MetalMom's python/metalmom/_native.py).

The declarations are read from ``include/metalmom.h`` so the Python binding and
the C header cannot drift apart.  There is no fallback: if the library is
missing the import fails with a RuntimeError naming the build command.
"""

import os
import re

import cffi

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
HEADER = os.path.join(_ROOT, "include", "metalmom.h")
LIB_PATH = os.path.join(_HERE, "_lib", "libmetalmom.so")


def header_cdef(path: str = HEADER) -> str:
    """The header's declarations in a form cffi's cdef accepts."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out, skip = [], []
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#if"):
            drop = "__cplusplus" in s or "MM_BUILDING_LIBRARY" in s
            skip.append(drop)
            continue
        if s.startswith("#else"):
            if skip:
                skip[-1] = True
            continue
        if s.startswith("#endif"):
            if skip:
                skip.pop()
            continue
        if any(skip):
            continue
        if s.startswith("#define"):
            if re.match(r"#define\s+MM_\w+\s+-?\d+\s*$", s):
                out.append(s)
            continue
        if s.startswith("#include"):
            continue
        out.append(line.replace("MM_API ", ""))
    return "\n".join(out)


def exported_names(path: str = HEADER):
    """Function names declared in the header."""
    return re.findall(r"\b(mm_\w+)\s*\(", header_cdef(path))


ffi = cffi.FFI()
ffi.cdef(header_cdef())

if not os.path.exists(LIB_PATH):
    raise RuntimeError(
        f"libmetalmom.so not found at {LIB_PATH}. "
        "Build it with `python metalmom_b200/build.py`.")

lib = ffi.dlopen(LIB_PATH)
