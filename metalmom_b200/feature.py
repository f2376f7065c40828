"""Mel spectrogram, MFCC and dB scaling (mirrors MetalMom python/metalmom/feature.py).

Same names, defaults (hop 512, as librosa), argument meaning and error
behaviour (RuntimeError "... failed with status N") as the reference wrappers
(feature.py:8-91, 94-167, 170-270); the computation runs in libmetalmom.so on
the GPU.
"""

import numpy as np

from ._buffer import buffer_to_numpy
from ._native import ffi, lib


def _call(name, fn, *args):
    ctx = lib.mm_init()
    if ctx == ffi.NULL:
        raise RuntimeError("Failed to initialize MetalMom context")
    try:
        out = ffi.new("MMBuffer*")
        status = fn(ctx, *args, out)
        if status != 0:
            raise RuntimeError(f"{name} failed with status {status}")
        return buffer_to_numpy(out)
    finally:
        lib.mm_destroy(ctx)


def melspectrogram(y=None, sr=22050, S=None, n_fft=2048, hop_length=None, win_length=None,
                   center=True, power=2.0, n_mels=128, fmin=0.0, fmax=None, **kwargs):
    """Mel spectrogram (n_mels, n_frames) of audio ``y``."""
    if S is not None:
        raise NotImplementedError("melspectrogram(S=...) is not served by the GPU front end")
    if y is None:
        raise ValueError("Either y or S must be provided")
    y = np.ascontiguousarray(y, dtype=np.float32)
    hop = hop_length if hop_length is not None else 512
    win = win_length if win_length is not None else n_fft
    c_fmax = float(fmax) if fmax is not None else 0.0
    ptr = ffi.cast("const float*", y.ctypes.data)
    return _call("mm_mel_spectrogram", lib.mm_mel_spectrogram, ptr, len(y), sr, n_fft, hop, win,
                 1 if center else 0, power, n_mels, fmin, c_fmax)


def mfcc(y=None, sr=22050, S=None, n_mfcc=20, n_fft=2048, hop_length=None, win_length=None,
         n_mels=128, fmin=0.0, fmax=None, center=True, **kwargs):
    """MFCCs (min(n_mfcc, n_mels), n_frames) of audio ``y``."""
    if S is not None:
        raise NotImplementedError("mfcc(S=...) is not served by the GPU front end")
    if y is None:
        raise ValueError("Either y or S must be provided")
    y = np.ascontiguousarray(y, dtype=np.float32)
    hop = hop_length if hop_length is not None else 512
    win = win_length if win_length is not None else n_fft
    c_fmax = float(fmax) if fmax is not None else 0.0
    ptr = ffi.cast("const float*", y.ctypes.data)
    return _call("mm_mfcc", lib.mm_mfcc, ptr, len(y), sr, n_mfcc, n_fft, hop, win, n_mels, fmin,
                 c_fmax, 1 if center else 0)


def _db(name, fn, S, ref, amin, top_db):
    S = np.ascontiguousarray(S, dtype=np.float32)
    shape = S.shape
    if callable(ref):
        ref = float(ref(S))
    flat = S.ravel()
    c_top_db = float(top_db) if top_db is not None else 0.0
    ptr = ffi.cast("const float*", flat.ctypes.data)
    return _call(name, fn, ptr, len(flat), ref, amin, c_top_db).reshape(shape)


def power_to_db(S, ref=1.0, amin=1e-10, top_db=80.0):
    """``10 log10(max(S, amin) / ref)`` floored at ``max - top_db``."""
    return _db("mm_power_to_db", lib.mm_power_to_db, S, ref, amin, top_db)


def amplitude_to_db(S, ref=1.0, amin=1e-5, top_db=80.0):
    """``20 log10(max(S, amin) / ref)`` floored at ``max - top_db``."""
    return _db("mm_amplitude_to_db", lib.mm_amplitude_to_db, S, ref, amin, top_db)


def delta(data, width=9, order=1, axis=-1, **kwargs):
    """Savitzky-Golay delta of order ``order`` along time of (n_features, n_frames)
    (mirrors feature.py:1312-1357 of the reference)."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    if data.ndim == 1:
        data = data.reshape(1, -1)
    n_features, n_frames = data.shape
    flat = data.ravel()
    ptr = ffi.cast("const float*", flat.ctypes.data)
    return _call("mm_delta", lib.mm_delta, ptr, len(flat), n_features, n_frames, width, order)


def stack_memory(data, n_steps=2, delay=1, **kwargs):
    """Stacked delayed copies (n_features * n_steps, n_frames), zeros before the
    start (mirrors feature.py:1360-1404 of the reference)."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    if data.ndim == 1:
        data = data.reshape(1, -1)
    n_features, n_frames = data.shape
    flat = data.ravel()
    ptr = ffi.cast("const float*", flat.ctypes.data)
    return _call("mm_stack_memory", lib.mm_stack_memory, ptr, len(flat), n_features, n_frames,
                 n_steps, delay)
