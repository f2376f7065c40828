"""ctypes front end for ``librefcpu.so`` (test infrastructure only).

The float32 C restatement of MetalMom's CPU path (see ``refcpu.c``): used as
the timed CPU baseline and as a second checker.
"""

import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = ctypes.CDLL(path)
        L.refcpu_n_frames.restype = ctypes.c_int64
        L.refcpu_n_frames.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.refcpu_mfcc.restype = ctypes.c_int
        L.refcpu_mfcc.argtypes = [ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_int] * 6 + [
            ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
            ctypes.c_void_p, ctypes.c_void_p]
        L.refcpu_stft.restype = ctypes.c_int
        L.refcpu_stft.argtypes = [ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_int] * 5 + [ctypes.c_void_p]
        L.refcpu_mfcc_batch.restype = ctypes.c_int
        L.refcpu_mfcc_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int] + [
            ctypes.c_int] * 6 + [ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                 ctypes.c_void_p, ctypes.c_int]
        _lib = L
    return _lib


def n_frames(L, n_fft, hop, center):
    return int(lib().refcpu_n_frames(L, n_fft, hop, 1 if center else 0))


def mfcc(y, sr=22050, n_mfcc=20, n_fft=2048, hop=512, win=None, n_mels=128, fmin=0.0,
         fmax=0.0, center=True, top_db=80.0, want_mel_db=False):
    y = np.ascontiguousarray(y, dtype=np.float32)
    win = n_fft if win is None else win
    T = n_frames(len(y), n_fft, hop, center)
    K = min(n_mfcc, n_mels)
    out = np.zeros((K, T), np.float32)
    mel = np.zeros((n_mels, T), np.float32) if want_mel_db else None
    rc = lib().refcpu_mfcc(y.ctypes.data, len(y), sr, n_mfcc, n_fft, hop, win, n_mels,
                           fmin, fmax or 0.0, 1 if center else 0, top_db,
                           out.ctypes.data, mel.ctypes.data if mel is not None else None)
    if rc != 0:
        raise RuntimeError("refcpu_mfcc failed")
    return (out, mel) if want_mel_db else out


def stft(y, n_fft=2048, hop=512, win=None, center=True, magnitude=True):
    y = np.ascontiguousarray(y, dtype=np.float32)
    win = n_fft if win is None else win
    T = n_frames(len(y), n_fft, hop, center)
    out = np.zeros((n_fft // 2 + 1, T), np.float32)
    rc = lib().refcpu_stft(y.ctypes.data, len(y), n_fft, hop, win, 1 if center else 0,
                           1 if magnitude else 0, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("refcpu_stft failed")
    return out


def mfcc_batch(clips, sr=22050, n_mfcc=20, n_fft=2048, hop=512, win=None, n_mels=128,
               fmin=0.0, fmax=0.0, center=True, top_db=80.0, n_threads=None):
    """MFCC of every clip, one clip per worker thread (all cores by default)."""
    clips = [np.ascontiguousarray(c, dtype=np.float32) for c in clips]
    win = n_fft if win is None else win
    n_threads = n_threads or os.cpu_count() or 1
    K = min(n_mfcc, n_mels)
    outs = [np.zeros((K, n_frames(len(c), n_fft, hop, center)), np.float32) for c in clips]
    n = len(clips)
    yp = (ctypes.c_void_p * n)(*[c.ctypes.data for c in clips])
    lp = (ctypes.c_int64 * n)(*[len(c) for c in clips])
    op = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
    rc = lib().refcpu_mfcc_batch(yp, lp, n, sr, n_mfcc, n_fft, hop, win, n_mels, fmin,
                                 fmax or 0.0, 1 if center else 0, top_db, op, n_threads)
    if rc != 0:
        raise RuntimeError("refcpu_mfcc_batch failed")
    return outs
