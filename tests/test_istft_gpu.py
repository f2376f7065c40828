"""Inverse STFT (mm_istft) against the FP64 oracle and as the inverse of the
forward transform (the reference's test_parity_istft.py round trips).

Tolerances: against the oracle, 1e-5 of the signal's peak where the
overlapped squared window sum is at least 1e-3, and the same bound on the
error times the window sum where it is smaller (at un-centred edges the sum
falls towards 1e-10 and dividing by it amplifies float32 rounding of the frame
sums, in the reference's float32 path as here); round trips within the
reference's 1e-3 and its energy ratio bound (0.99, 1.01).
"""

import numpy as np
import pytest

import metalmom_b200 as M
from metalmom_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_fft,hop,win,center,L,length", [
    (2048, 512, 2048, True, 22050, 22050),
    (2048, 512, 2048, True, 22050, None),
    (1024, 256, 1024, True, 8192, 8192),
    (512, 160, 400, True, 16000, 16000),     # window shorter than n_fft
    (2048, 441, 2048, False, 30001, None),   # odd hop, no centring
    (256, 64, 256, False, 4000, 5000),       # zero-padded to a longer length
    (4096, 1024, 4096, True, 50000, 50000),
    (16, 4, 16, True, 300, None),
])
def test_istft_vs_oracle(n_fft, hop, win, center, L, length):
    y = synth.music_clip(L, 22050, seed=L + n_fft)
    S = O.stft_complex(y, n_fft, hop, win, center).astype(np.complex64)
    got = M.istft(S, hop_length=hop, win_length=win, center=center, length=length)
    exp = O.istft(S, hop, win, center, length)
    assert got.shape == exp.shape and got.dtype == np.float32
    ws = _window_sum(n_fft, hop, win, S.shape[1], center, len(exp))
    err = np.abs(got - exp) * np.minimum(1.0, ws / 1e-3)
    assert err.max() <= 1e-5 * max(np.abs(exp).max(), 1.0)


def _window_sum(n_fft, hop, win, n_frames, center, n_out):
    """Overlapped squared synthesis window at each output sample."""
    w = O.prepare_window(win, n_fft)
    total = n_fft + (n_frames - 1) * hop
    ws = np.zeros(max(total, n_out + n_fft))
    for f in range(n_frames):
        ws[f * hop:f * hop + n_fft] += w * w
    start = n_fft // 2 if center else 0
    return ws[start:start + n_out]


def test_istft_round_trips():
    sr = 22050
    t = np.arange(sr) / sr
    y = (0.5 * np.sin(2 * np.pi * 440 * t) + 0.3 * np.sin(2 * np.pi * 880 * t)).astype(np.float32)
    S = O.stft_complex(y, 2048, 512, 2048, True).astype(np.complex64)
    np.testing.assert_allclose(M.istft(S, hop_length=512, length=len(y)), y, rtol=1e-3, atol=1e-3)
    rng = np.random.default_rng(123)
    y = rng.standard_normal(16384).astype(np.float32)
    S = O.stft_complex(y, 2048, 512, 2048, True).astype(np.complex64)
    r = M.istft(S, hop_length=512, length=len(y))
    ratio = np.sum(r.astype(np.float64) ** 2) / np.sum(y.astype(np.float64) ** 2)
    assert 0.99 < ratio < 1.01


def test_istft_edge_cases():
    S = np.zeros((1025, 3), np.complex64)
    assert M.istft(S, hop_length=512).shape == (1024,)
    odd = np.ones((7, 4), np.complex64)  # n_fft 12: not a power of two -> zeros
    r = M.istft(odd, hop_length=3, center=False)
    assert r.shape == (12 + 3 * 3,) and np.all(r == 0)
    with pytest.raises(RuntimeError, match="status -1"):
        M.istft(S, hop_length=0)
