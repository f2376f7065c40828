"""``stft`` and ``istft`` (mirror MetalMom python/metalmom/core.py:198-319)."""

import numpy as np

from ._bridge import bridge_call, float_ptr, stft_params
from ._native import lib

SR_UNUSED = 22050  # the bridge's STFT entry points take a sample rate they do not use


def _defaults(n_fft, hop_length, win_length):
    return (hop_length if hop_length is not None else n_fft // 4,
            win_length if win_length is not None else n_fft)


def stft(y, n_fft=2048, hop_length=None, win_length=None, center=True):
    """Magnitude STFT, shape (n_fft // 2 + 1, n_frames), computed on the GPU.

    Defaults as MetalMom's ``core.stft``: hop ``n_fft // 4``, window ``n_fft``,
    sample rate 22050 passed to the bridge (core.py:223-243).
    """
    y, ptr = float_ptr(y)
    hop, win = _defaults(n_fft, hop_length, win_length)
    return bridge_call("mm_stft", lib.mm_stft, ptr, len(y), SR_UNUSED, stft_params(n_fft, hop, win, center))


def stft_complex(y, n_fft=2048, hop_length=None, win_length=None, center=True):
    """Complex STFT, complex64 (n_fft // 2 + 1, n_frames), computed on the GPU.

    The Python form of MetalMom's ``STFT.computeComplex``
    (Sources/MetalMomCore/Spectral/STFT.swift:512-668): zero centre padding,
    hop ``n_fft // 4`` and window ``n_fft`` by default, DC and Nyquist real.
    ``istft(stft_complex(y))`` reconstructs ``y``.
    """
    y, ptr = float_ptr(y)
    hop, win = _defaults(n_fft, hop_length, win_length)
    inter = bridge_call("mm_stft_complex", lib.mm_stft_complex, ptr, len(y), SR_UNUSED,
                        stft_params(n_fft, hop, win, center))  # [n_freqs, n_frames, 2] float32
    return np.ascontiguousarray(inter).view(np.complex64)[..., 0]


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
    hop, win = _defaults(n_fft, hop_length, win_length)
    inter, ptr = float_ptr(np.ascontiguousarray(stft_matrix).view(np.float32))
    return bridge_call("mm_istft", lib.mm_istft, ptr, inter.size, n_freqs, n_frames, SR_UNUSED, hop, win,
                       1 if center else 0, length if length is not None else 0)
