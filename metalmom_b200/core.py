"""``stft`` (mirrors MetalMom python/metalmom/core.py:198-250)."""

import numpy as np

from ._buffer import buffer_to_numpy
from ._native import ffi, lib


def stft(y, n_fft=2048, hop_length=None, win_length=None, center=True):
    """Magnitude STFT, shape (n_fft // 2 + 1, n_frames), computed on the GPU.

    Defaults as MetalMom's ``core.stft``: hop ``n_fft // 4``, window ``n_fft``,
    sample rate 22050 passed to the bridge (core.py:223-243).
    """
    y = np.ascontiguousarray(y, dtype=np.float32)
    hop = hop_length if hop_length is not None else n_fft // 4
    win = win_length if win_length is not None else n_fft
    ctx = lib.mm_init()
    if ctx == ffi.NULL:
        raise RuntimeError("Failed to initialize MetalMom context")
    try:
        params = ffi.new("MMSTFTParams*")
        params.n_fft = n_fft
        params.hop_length = hop
        params.win_length = win
        params.center = 1 if center else 0
        out = ffi.new("MMBuffer*")
        ptr = ffi.cast("const float*", y.ctypes.data)
        status = lib.mm_stft(ctx, ptr, len(y), 22050, params, out)
        if status != 0:
            raise RuntimeError(f"mm_stft failed with status {status}")
        return buffer_to_numpy(out)
    finally:
        lib.mm_destroy(ctx)
