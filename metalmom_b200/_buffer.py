"""MMBuffer -> NumPy (mirrors MetalMom's python/metalmom/_buffer.py semantics).

The data is copied out and the C buffer is always freed, even if the copy or
reshape raises.
"""

import numpy as np

from ._native import ffi, lib


def buffer_to_numpy(buf):
    if buf.data == ffi.NULL or buf.count == 0:
        shape = tuple(buf.shape[i] for i in range(buf.ndim))
        lib.mm_buffer_free(buf)
        return np.empty(shape, dtype=np.float32)
    try:
        count = buf.count
        data = np.frombuffer(ffi.buffer(buf.data, count * 4), dtype=np.float32).copy()
        shape = tuple(buf.shape[i] for i in range(buf.ndim))
        return data.reshape(shape)
    finally:
        lib.mm_buffer_free(buf)


def numpy_to_float_ptr(arr):
    arr = np.ascontiguousarray(arr, dtype=np.float32)
    return ffi.cast("const float*", arr.ctypes.data), len(arr)
