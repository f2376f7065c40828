"""Calling the C ABI from Python: one context per call, the library-owned
output buffer copied into NumPy and released, and a RuntimeError naming the
entry point and its status on failure (the error behaviour of MetalMom's
Python wrappers, which build a context per call as well)."""

import numpy as np

from ._native import ffi, lib


def take_buffer(buf):
    """The floats of a filled MMBuffer as a new array of its shape; the C
    buffer is released whatever happens (an empty result has data NULL and
    count 0 with the shape set)."""
    try:
        shape = tuple(int(buf.shape[d]) for d in range(buf.ndim))
        n = int(buf.count)
        if n == 0 or buf.data == ffi.NULL:
            return np.empty(shape, dtype=np.float32)
        view = np.frombuffer(ffi.buffer(buf.data, 4 * n), dtype=np.float32)
        return view.reshape(shape).copy()
    finally:
        lib.mm_buffer_free(buf)


def bridge_call(name, fn, *args):
    """fn(ctx, *args, out) inside a fresh context; the output as an array."""
    ctx = lib.mm_init()
    if ctx == ffi.NULL:
        raise RuntimeError("Failed to initialize MetalMom context")
    try:
        out = ffi.new("MMBuffer*")
        status = fn(ctx, *args, out)
        if status != 0:
            raise RuntimeError(f"{name} failed with status {status}")
        return take_buffer(out)
    finally:
        lib.mm_destroy(ctx)


def float_ptr(a):
    """A contiguous float32 view of `a` and its cffi pointer (keep the view
    alive while the pointer is in use)."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, ffi.cast("const float*", a.ctypes.data)


def stft_params(n_fft, hop, win, center):
    p = ffi.new("MMSTFTParams*")
    p.n_fft, p.hop_length, p.win_length, p.center = n_fft, hop, win, 1 if center else 0
    return p
