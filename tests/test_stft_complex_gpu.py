"""Complex STFT (mm_stft_complex, the C-ABI form of STFT.computeComplex in
Sources/MetalMomCore/Spectral/STFT.swift:512-668) against the FP64 oracle,
the magnitude golden, and as the forward half of the iSTFT round trip.

Tolerances: |X_gpu - X_oracle| <= 2e-5 of the largest |X| of the clip (the
float32 FFT bound of the magnitude tests); the round trip within the
reference's 1e-3 (test_parity_istft.py).
"""

import numpy as np
import pytest

import metalmom_b200 as M
from metalmom_b200 import synth
from metalmom_b200._native import ffi, lib
from oracle import oracle as O

from goldens import golden, signal_440

pytestmark = pytest.mark.gpu


def _check(got, exp):
    assert got.shape == exp.shape and got.dtype == np.complex64
    if exp.size:
        assert np.abs(got - exp).max() <= 2e-5 * max(np.abs(exp).max(), 1e-30)
        # DC and Nyquist are real, as in the reference's packed format
        assert np.all(got[0].imag == 0) and np.all(got[-1].imag == 0)


@pytest.mark.parametrize("n_fft", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 32768])
def test_stft_complex_all_sizes_vs_oracle(n_fft):
    rng = np.random.default_rng(n_fft + 11)
    L = max(3 * n_fft + 17, 64)
    y = rng.standard_normal(L).astype(np.float32)
    hop = max(1, n_fft // 4)
    got = M.stft_complex(y, n_fft=n_fft, hop_length=hop)
    exp = O.stft_complex(y, n_fft, hop, n_fft, True)
    assert got.shape == (n_fft // 2 + 1, O.n_frames(L, n_fft, hop, True))
    _check(got, exp)


@pytest.mark.parametrize("n_fft,hop,win,center,L", [
    (2048, 512, 2048, True, 661500 // 10),
    (2048, 512, 2048, False, 50000),
    (512, 160, 400, True, 16000),      # window shorter than n_fft
    (2048, 512, 4096, True, 22050),    # window longer than n_fft
    (1024, 4096, 1024, True, 22050),   # hop longer than n_fft
    (2048, 441, 2048, True, 30001),    # odd hop: unaligned frame starts
    (2048, 512, 2048, False, 2048),    # exactly one frame
])
def test_stft_complex_cases_vs_oracle(n_fft, hop, win, center, L):
    y = synth.music_clip(L, 22050, seed=L + n_fft + 3)
    _check(M.stft_complex(y, n_fft=n_fft, hop_length=hop, win_length=win, center=center),
           O.stft_complex(y, n_fft, hop, win, center))


def test_stft_complex_magnitude_golden():
    y = signal_440()
    X = M.stft_complex(y, n_fft=2048, hop_length=512)
    np.testing.assert_allclose(np.abs(X), golden("stft_440hz_default_magnitude"), rtol=1e-4, atol=1e-4)
    # the magnitude entry point and the complex one agree
    np.testing.assert_allclose(np.abs(X), M.stft(y, n_fft=2048, hop_length=512), rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("n_fft,hop,L", [(2048, 512, 22050), (1024, 256, 8192), (512, 128, 16000)])
def test_stft_complex_istft_round_trip(n_fft, hop, L):
    y = synth.music_clip(L, 22050, seed=n_fft)
    back = M.istft(M.stft_complex(y, n_fft=n_fft, hop_length=hop), hop_length=hop, length=L)
    np.testing.assert_allclose(back, y, atol=1e-3)
    ratio = np.sum(back.astype(np.float64) ** 2) / np.sum(y.astype(np.float64) ** 2)
    assert 0.99 < ratio < 1.01


def test_stft_complex_edge_shapes_and_errors():
    y = np.ones(1000, np.float32)
    # non-power-of-two n_fft: empty [n_freqs, 0], as computeComplex returns
    X = M.stft_complex(y, n_fft=1000, hop_length=250)
    assert X.shape == (501, 0)
    # shorter than one frame without centring: no frames
    assert M.stft_complex(y[:100], n_fft=256, hop_length=64, center=False).shape == (129, 0)
    ctx = lib.mm_init()
    try:
        p = ffi.new("MMSTFTParams*")
        p.n_fft, p.hop_length, p.win_length, p.center = 2048, 512, 2048, 1
        out = ffi.new("MMBuffer*")
        ptr = ffi.cast("const float*", y.ctypes.data)
        assert lib.mm_stft_complex(ffi.NULL, ptr, len(y), 22050, p, out) == -1
        assert lib.mm_stft_complex(ctx, ffi.NULL, len(y), 22050, p, out) == -1
        assert lib.mm_stft_complex(ctx, ptr, 0, 22050, p, out) == -1
        p.n_fft = 0
        assert lib.mm_stft_complex(ctx, ptr, len(y), 22050, p, out) == -1
        # hop / win sentinels: <= 0 take n_fft // 4 and n_fft
        p.n_fft, p.hop_length, p.win_length = 256, 0, 0
        assert lib.mm_stft_complex(ctx, ptr, len(y), 22050, p, out) == 0
        assert out.ndim == 3 and out.shape[0] == 129 and out.shape[2] == 2
        assert out.shape[1] == O.n_frames(len(y), 256, 64, True) and out.count == 2 * 129 * out.shape[1]
        lib.mm_buffer_free(out)
    finally:
        lib.mm_destroy(ctx)
