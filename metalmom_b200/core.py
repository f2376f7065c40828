"""``stft`` and ``istft`` (mirror MetalMom python/metalmom/core.py:198-319)."""

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


def stft_complex(y, n_fft=2048, hop_length=None, win_length=None, center=True):
    """Complex STFT, complex64 (n_fft // 2 + 1, n_frames), computed on the GPU.

    The Python form of MetalMom's ``STFT.computeComplex``
    (Sources/MetalMomCore/Spectral/STFT.swift:512-668): zero centre padding,
    hop ``n_fft // 4`` and window ``n_fft`` by default, DC and Nyquist real.
    ``istft(stft_complex(y))`` reconstructs ``y``.
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
        status = lib.mm_stft_complex(ctx, ptr, len(y), 22050, params, out)
        if status != 0:
            raise RuntimeError(f"mm_stft_complex failed with status {status}")
        inter = buffer_to_numpy(out)  # [n_freqs, n_frames, 2] float32
        return np.ascontiguousarray(inter).view(np.complex64)[..., 0]
    finally:
        lib.mm_destroy(ctx)


def istft(stft_matrix, hop_length=None, win_length=None, center=True, length=None):
    """Inverse STFT of a complex spectrogram (n_fft // 2 + 1, n_frames), computed on
    the GPU (mirrors MetalMom python/metalmom/core.py:253-319: hop ``n_fft // 4``,
    window ``n_fft``, 1-D float32 result)."""
    if not np.iscomplexobj(stft_matrix):
        stft_matrix = np.asarray(stft_matrix).astype(np.complex64)
    else:
        stft_matrix = np.asarray(stft_matrix, dtype=np.complex64)
    n_freqs, n_frames = stft_matrix.shape
    n_fft = (n_freqs - 1) * 2
    hop = hop_length if hop_length is not None else n_fft // 4
    win = win_length if win_length is not None else n_fft
    inter = np.ascontiguousarray(stft_matrix).view(np.float32)
    ctx = lib.mm_init()
    if ctx == ffi.NULL:
        raise RuntimeError("Failed to initialize MetalMom context")
    try:
        out = ffi.new("MMBuffer*")
        ptr = ffi.cast("const float*", inter.ctypes.data)
        status = lib.mm_istft(ctx, ptr, inter.size, n_freqs, n_frames, 22050, hop, win,
                              1 if center else 0, length if length is not None else 0, out)
        if status != 0:
            raise RuntimeError(f"mm_istft failed with status {status}")
        return buffer_to_numpy(out)
    finally:
        lib.mm_destroy(ctx)
