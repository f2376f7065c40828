"""Spectrogram-input operations on the GPU: melspectrogram(S=...) and
mfcc(S=...) (the reference's feature.py:50-57 and 130-134, which run numpy /
scipy there) and dB scaling of device buffers (ref given or ref=np.max taken
on the device).

Tolerances: mel projection within 1e-5 of the largest band value of the clip
(float32 sums of <= 1025 products against float64); DCT within 1e-5 of the
largest |coefficient|; the goldens at the reference's rtol = atol = 1e-4; the
device dB path bitwise equal to the host dB path (same kernels).
"""

import numpy as np
import pytest
import torch

import metalmom_b200 as M
from metalmom_b200 import synth
from oracle import oracle as O

from goldens import golden, signal_440

pytestmark = pytest.mark.gpu
SR = 22050


def _close(got, exp, tol=1e-5):
    assert got.shape == exp.shape and got.dtype == np.float32
    if exp.size:
        assert np.abs(got - exp).max() <= tol * max(np.abs(exp).max(), 1e-30)


@pytest.mark.parametrize("n_fft,n_mels,fmin,fmax,T", [
    (2048, 128, 0.0, None, 431),
    (1024, 40, 0.0, None, 100),
    (2048, 64, 300.0, 8000.0, 77),
    (512, 80, 20.0, 8000.0, 1001),
    (1000, 32, 0.0, None, 12),      # n_fft need not be a power of two here
    (2048, 128, 0.0, None, 1),
])
def test_mel_project_vs_oracle(n_fft, n_mels, fmin, fmax, T):
    rng = np.random.default_rng(n_fft + T)
    S = (rng.random((n_fft // 2 + 1, T)) ** 3).astype(np.float32)
    got = M.melspectrogram(S=S, sr=SR, n_fft=n_fft, n_mels=n_mels, fmin=fmin, fmax=fmax)
    _close(got, O.mel_project(S, SR, n_fft, n_mels, fmin, fmax))


def test_mel_project_golden_and_native_agree():
    y = signal_440()
    P = M.stft(y, n_fft=2048, hop_length=512) ** 2
    got = M.melspectrogram(S=P, sr=SR)
    np.testing.assert_allclose(got, golden("mel_spectrogram_440hz_default"), rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(got, M.melspectrogram(y=y, sr=SR), rtol=1e-4, atol=1e-6)


def test_mel_project_shapes_and_nonfinite_columns():
    rng = np.random.default_rng(1)
    S = rng.random((1025, 6)).astype(np.float32)
    S[7, 2] = np.inf
    S[100, 4] = np.nan
    got = M.melspectrogram(S=S, sr=SR)
    with np.errstate(invalid="ignore"):  # 0 * inf in the float64 product, as intended
        exp = O.mel_project(S, SR)
    assert np.all(np.isnan(got[:, 2])) and np.all(np.isnan(got[:, 4]))
    ok = [0, 1, 3, 5]
    _close(got[:, ok], exp[:, ok])
    # 1-D: one frame
    v = M.melspectrogram(S=S[:, 0], sr=SR)
    assert v.shape == (128,)
    _close(v, exp[:, 0])
    # batched [..., n_freqs, n_frames], as numpy's matmul broadcasts
    B = rng.random((3, 2, 1025, 5)).astype(np.float32)
    gb = M.melspectrogram(S=B, sr=SR)
    assert gb.shape == (3, 2, 128, 5)
    _close(gb, np.stack([np.stack([O.mel_project(B[i, j], SR) for j in range(2)]) for i in range(3)]))
    assert M.melspectrogram(S=S, sr=SR, n_mels=0).shape == (0, 6)


@pytest.mark.parametrize("rows,T,n_mfcc", [(128, 431, 20), (40, 100, 13), (64, 7, 20), (20, 33, 40),
                                           (128, 1, 20), (13, 50, -3)])
def test_dct_ortho_vs_oracle(rows, T, n_mfcc):
    rng = np.random.default_rng(rows * 7 + T)
    S = (rng.standard_normal((rows, T)) * 20 - 40).astype(np.float32)
    got = M.mfcc(S=S, n_mfcc=n_mfcc)
    k = len(range(rows)[:n_mfcc])
    _close(got, O.dct_ortho(S, k))


def test_dct_ortho_golden_and_shapes():
    y = signal_440()
    C = M.mfcc(S=M.power_to_db(M.melspectrogram(y=y, sr=SR)), n_mfcc=20)
    np.testing.assert_allclose(C, golden("mfcc_440hz_default"), rtol=1e-4, atol=1e-4)
    rng = np.random.default_rng(5)
    v = rng.standard_normal(40).astype(np.float32)
    c1 = M.mfcc(S=v, n_mfcc=13)
    assert c1.shape == (13,)
    _close(c1, O.dct_ortho(v[:, None], 13)[:, 0])
    B = rng.standard_normal((40, 2, 6)).astype(np.float32)   # scipy's dct along axis 0 of a 3-D array
    cb = M.mfcc(S=B, n_mfcc=13)
    assert cb.shape == (13, 2, 6)
    _close(cb, O.dct_ortho(B.reshape(40, -1), 13).reshape(13, 2, 6))


@pytest.mark.parametrize("fn_dev,fn_host,amin", [(M.power_to_db_device, M.power_to_db, 1e-10),
                                                 (M.amplitude_to_db_device, M.amplitude_to_db, 1e-5)])
@pytest.mark.parametrize("ref", [1.0, 0.25, np.max])
def test_db_device_matches_host(fn_dev, fn_host, amin, ref):
    S = (np.random.default_rng(9).random((257, 300)) ** 4).astype(np.float32)
    S[3, 4] = 0.0
    exp = fn_host(S, ref=ref, amin=amin, top_db=80.0)
    x = torch.from_numpy(S).cuda()
    got = fn_dev(x, ref=ref, amin=amin, top_db=80.0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), exp)
    # in place, no floor
    fn_dev(x, ref=ref, amin=amin, top_db=None, out=x)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(x.cpu().numpy(), fn_host(S, ref=ref, amin=amin, top_db=None))


def test_db_device_ref_max_with_nan_is_nan():
    S = np.ones((4, 5), np.float32)
    S[1, 1] = np.nan
    x = torch.from_numpy(S).cuda()
    got = M.power_to_db_device(x, ref=np.max, top_db=None)
    torch.cuda.synchronize()
    assert torch.isnan(got).all()  # np.max of an array with NaN is NaN
