"""Onset strength (mirrors MetalMom python/metalmom/onset.py:8-71).

Same name, defaults and return shapes: (n_frames,) when ``aggregate`` else
(n_mels, n_frames).  The log-mel rows come from the GPU front end and the
spectral flux is a kernel on the device.
"""

import numpy as np

from .feature import _call
from ._native import ffi, lib


def onset_strength(y=None, sr=22050, S=None, n_fft=2048, hop_length=512, n_mels=128, fmin=0.0,
                   fmax=None, center=True, aggregate=True, **kwargs):
    if S is not None:
        raise NotImplementedError("onset_strength(S=...) is not served by the GPU front end")
    if y is None:
        raise ValueError("y must be provided")
    y = np.ascontiguousarray(y, dtype=np.float32)
    c_fmax = float(fmax) if fmax is not None else 0.0
    ptr = ffi.cast("const float*", y.ctypes.data)
    res = _call("mm_onset_strength", lib.mm_onset_strength, ptr, len(y), sr, n_fft, hop_length, n_mels,
                fmin, c_fmax, 1 if center else 0, 1 if aggregate else 0)
    return res.ravel() if aggregate else res
