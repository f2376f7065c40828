"""Mel spectrogram, MFCC and dB scaling (mirrors MetalMom python/metalmom/feature.py).

Same names, defaults (hop 512, as librosa), argument meaning and error
behaviour (RuntimeError "... failed with status N") as the reference wrappers
(feature.py:8-91, 94-167, 170-270); the computation runs in libmetalmom.so on
the GPU.
"""

import numpy as np

from ._bridge import bridge_call as _call
from ._native import ffi, lib


def _columns(S, rows_axis):
    """S as [rows, columns] float32 plus a function restoring the other axes.

    rows_axis -2: numpy matmul semantics, [..., rows, frames] (the filterbank
    product); 0: scipy ``dct(axis=0)`` semantics, [rows, ...].
    """
    S = np.ascontiguousarray(S, dtype=np.float32)  # 0-d becomes shape (1,), as in numpy
    if S.ndim == 1:
        return S.reshape(-1, 1), lambda r: r.reshape(r.shape[0])
    if S.ndim == 2:
        return S, lambda r: r
    if rows_axis == 0:
        rest = S.shape[1:]
        return S.reshape(S.shape[0], -1), lambda r: r.reshape((r.shape[0],) + rest)
    lead, (rows, frames) = S.shape[:-2], S.shape[-2:]
    flat = np.ascontiguousarray(np.moveaxis(S, -2, 0)).reshape(rows, -1)
    return flat, lambda r: np.moveaxis(r.reshape((r.shape[0],) + lead + (frames,)), 0, -2)


def _mel_project(S, sr, n_fft, n_mels, fmin, fmax):
    S = np.ascontiguousarray(S, dtype=np.float32)
    n_freqs = n_fft // 2 + 1
    rows_axis = 0 if S.ndim == 1 else -2
    if S.shape[rows_axis] != n_freqs:
        raise ValueError(f"matmul: S has {S.shape[rows_axis]} frequency rows, the mel filterbank of "
                         f"n_fft={n_fft} expects {n_freqs}")
    flat, restore = _columns(S, -2)
    c_fmax = float(fmax) if fmax is not None else 0.0
    ptr = ffi.cast("const float*", flat.ctypes.data)
    r = _call("mm_mel_project", lib.mm_mel_project, ptr, flat.size, flat.shape[0], flat.shape[1], sr, n_fft,
              n_mels, float(fmin), c_fmax)
    return restore(r)


def _dct_ortho(S, n_mfcc):
    flat, restore = _columns(S, 0)
    n_out = len(range(flat.shape[0])[:n_mfcc])  # numpy slice semantics of [:n_mfcc]
    ptr = ffi.cast("const float*", flat.ctypes.data)
    r = _call("mm_dct_ortho", lib.mm_dct_ortho, ptr, flat.size, flat.shape[0], flat.shape[1], n_out)
    return restore(r)


def melspectrogram(y=None, sr=22050, S=None, n_fft=2048, hop_length=None, win_length=None,
                   center=True, power=2.0, n_mels=128, fmin=0.0, fmax=None, **kwargs):
    """Mel spectrogram (n_mels, n_frames) of audio ``y``, or of a given
    spectrogram ``S`` (the filterbank applied to S as given, as the reference's
    feature.py:50-57; ``power`` is not applied), on the GPU."""
    if S is not None:
        return _mel_project(S, sr, n_fft, n_mels, fmin, fmax)
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
    """MFCCs (min(n_mfcc, n_mels), n_frames) of audio ``y``, or the DCT-II
    ortho along axis 0 of a given log-mel spectrogram ``S``, first ``n_mfcc``
    rows (the reference's feature.py:130-134), on the GPU."""
    if S is not None:
        return _dct_ortho(S, n_mfcc)
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


def _device_ptr(x):
    """(address, element count) of a float32 CUDA tensor or an (address, count) pair."""
    if isinstance(x, tuple):
        return int(x[0]), int(x[1])
    if not (x.is_cuda and x.dtype.is_floating_point and x.element_size() == 4 and x.is_contiguous()):
        raise ValueError("expected a contiguous float32 CUDA tensor")
    return x.data_ptr(), x.numel()


def _db_device(name, fn, x, ref, amin, top_db, out, stream):
    src, n = _device_ptr(x)
    if out is None:
        out = x.new_empty(x.shape) if not isinstance(x, tuple) else x
    dst, n_out = _device_ptr(out)
    if n_out != n:
        raise ValueError("out must have as many elements as the input")
    ref_mode, ref_val = 0, 1.0
    if ref is np.max or ref is max or (isinstance(ref, str) and ref == "max"):
        ref_mode = 1
    elif callable(ref):
        ref_val = float(ref(x))
    else:
        ref_val = float(ref)
    if stream is None:
        import torch
        stream = torch.cuda.current_stream().cuda_stream
    c_top_db = float(top_db) if top_db is not None else 0.0
    st = fn(ffi.cast("const float*", src), n, ref_val, ref_mode, float(amin), c_top_db,
            ffi.cast("float*", dst), ffi.cast("void*", int(stream)))
    if st != 0:
        raise RuntimeError(f"{name} failed with status {st}")
    return out


def power_to_db_device(x, ref=1.0, amin=1e-10, top_db=80.0, out=None, stream=None):
    """``power_to_db`` of a CUDA tensor on its stream, without a host copy;
    ``ref=np.max`` takes the maximum on the device.  ``out=x`` works in place."""
    return _db_device("mm_power_to_db_device", lib.mm_power_to_db_device, x, ref, amin, top_db, out, stream)


def amplitude_to_db_device(x, ref=1.0, amin=1e-5, top_db=80.0, out=None, stream=None):
    """``amplitude_to_db`` of a CUDA tensor (20 log10), as ``power_to_db_device``."""
    return _db_device("mm_amplitude_to_db_device", lib.mm_amplitude_to_db_device, x, ref, amin, top_db, out,
                      stream)


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
