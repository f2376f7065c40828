"""Pin the CPU oracle against the reference's golden vectors.

Mirrors MetalMom's ``Tests/test_parity_{stft,melspec,mfcc,mel_filterbank,
scaling}.py`` cases and tolerances, with the oracle in place of the native
library.  If the oracle matches these goldens, parity of the CUDA path against
the oracle is parity against the reference's pinned outputs.
"""

import numpy as np
import pytest

from goldens import golden, signal_440
from oracle import oracle as O

SR = 22050


def test_signal_fixture():
    y = signal_440()
    assert y.shape == (22050,) and y.dtype == np.float32


def test_stft_magnitude_golden():
    """test_parity_stft.py:38-49 (rtol=atol=1e-4)."""
    y = signal_440()
    exp = golden("stft_440hz_default_magnitude")
    got = O.stft_magnitude(y, 2048, 512, 2048, True)
    assert got.shape == exp.shape == (1025, 44)
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4)
    mid = got.shape[1] // 2
    assert np.argmax(got[:, mid]) == np.argmax(exp[:, mid])
    ratio = np.sum(got ** 2) / np.sum(exp.astype(np.float64) ** 2)
    assert 0.99 < ratio < 1.01


def test_reflect_padding_is_not_the_reference():
    """The goldens were made with zero padding; reflect must differ."""
    y = signal_440()
    exp = golden("stft_440hz_default_magnitude")
    got = O.stft_magnitude(y, 2048, 512, 2048, True, pad_mode=O.PAD_REFLECT)
    assert np.max(np.abs(got - exp)) > 1.0


@pytest.mark.parametrize("name,kw", [
    ("mel_filterbank_128_2048", dict(sr=SR, n_fft=2048, n_mels=128)),
    ("mel_filterbank_40_1024", dict(sr=SR, n_fft=1024, n_mels=40)),
    ("mel_filterbank_64_2048_300_8000", dict(sr=SR, n_fft=2048, n_mels=64, fmin=300, fmax=8000)),
])
def test_mel_filterbank_golden(name, kw):
    """test_parity_mel_filterbank.py:119-147 (rtol 1e-5, atol 1e-6)."""
    exp = golden(name)
    got = O.mel_filterbank(**kw)
    assert got.shape == exp.shape
    np.testing.assert_allclose(got, exp, rtol=1e-5, atol=1e-6)
    assert np.all(got >= 0)
    assert np.all(got.sum(axis=1) > 0)


@pytest.mark.parametrize("name,kw", [
    ("mel_spectrogram_440hz_default", dict()),
    ("mel_spectrogram_440hz_40_1024", dict(n_fft=1024, n_mels=40)),
    ("mel_spectrogram_440hz_64_fmin300_fmax8000", dict(n_fft=2048, n_mels=64, fmin=300, fmax=8000)),
])
def test_melspectrogram_golden(name, kw):
    """test_parity_melspec.py:78-118 (rtol=atol=1e-4); librosa hop is 512."""
    y = signal_440()
    exp = golden(name)
    got = O.melspectrogram(y, SR, hop=512, **kw)
    assert got.shape == exp.shape
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("name,kw,tol", [
    ("mfcc_440hz_default", dict(n_mfcc=20), 1e-4),
    ("mfcc_440hz_13_1024", dict(n_mfcc=13, n_fft=1024, n_mels=40), 1e-4),
    ("mfcc_440hz_20_64_fmin300_fmax8000", dict(n_mfcc=20, n_fft=2048, n_mels=64, fmin=300, fmax=8000), 5e-4),
])
def test_mfcc_golden(name, kw, tol):
    """test_parity_mfcc.py:78-120 (1e-4; 5e-4 for fmin=300/fmax=8000)."""
    y = signal_440()
    exp = golden(name)
    got = O.mfcc(y, SR, hop=512, **kw)
    assert got.shape == exp.shape
    np.testing.assert_allclose(got, exp, rtol=tol, atol=tol)


def test_power_to_db_ref_max_golden():
    """test_parity_scaling.py:58-75: power_to_db(S**2, ref=np.max)."""
    S = golden("stft_440hz_default_magnitude").astype(np.float32)
    P = S ** 2
    got = O.power_to_db(P, ref=float(np.max(P)))
    np.testing.assert_allclose(got, golden("stft_440hz_power_db"), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("ref_max,name", [(True, "stft_440hz_amplitude_db"),
                                          (False, "stft_440hz_amplitude_db_ref1")])
def test_amplitude_to_db_golden(ref_max, name):
    """test_parity_scaling.py:20-55."""
    S = golden("stft_440hz_default_magnitude").astype(np.float32)
    ref = float(np.max(S)) if ref_max else 1.0
    got = O.amplitude_to_db(S, ref=ref)
    np.testing.assert_allclose(got, golden(name), rtol=1e-4, atol=1e-4)


def test_frame_counts_sweep():
    """ParameterSweepTests.swift:35-98: frame counts over n_fft x hop x center x length."""
    for n_fft in (256, 512, 1024, 2048, 4096):
        for hop in (n_fft // 4, n_fft // 2):
            for center in (True, False):
                for L in (4096, 22050, 44100):
                    nf = O.n_frames(L, n_fft, hop, center)
                    padded = L + (n_fft if center else 0)
                    exp = 0 if padded < n_fft else 1 + (padded - n_fft) // hop
                    assert nf == exp
                    assert O.stft_power(np.zeros(L), n_fft, hop, n_fft, center).shape == (n_fft // 2 + 1, exp)


def test_edge_frame_counts():
    """EdgeCaseTests.swift:69-171 frame-count semantics."""
    assert O.n_frames(0, 2048, 512, True) == 1        # empty + center -> 1 frame
    assert O.n_frames(0, 2048, 512, False) == 0
    assert O.n_frames(1, 2048, 512, True) == 1
    assert O.n_frames(8000, 1000, 250, True) == 0     # non power of two
    assert O.n_frames(22050, 2048, 4096, True) == 1 + 22050 // 4096


def test_window_known_values():
    """WindowTests.swift: periodic Hann; short windows are centred in n_fft."""
    w = O.hann_periodic(4)
    np.testing.assert_allclose(w, [0.0, 0.5, 1.0, 0.5], atol=1e-15)
    full = O.prepare_window(400, 512)
    assert np.all(full[:56] == 0) and np.all(full[456:] == 0)
    np.testing.assert_allclose(full[56:456], O.hann_periodic(400))
    trunc = O.prepare_window(4096, 2048)
    np.testing.assert_allclose(trunc, O.hann_periodic(4096)[1024:3072])
    assert np.all(O.prepare_window(0, 64) == 0)


def test_dct_basis_orthonormal():
    """MFCCTests.swift:119: DCT-II ortho rows are orthonormal."""
    B = O.dct_basis(40, 40)
    np.testing.assert_allclose(B @ B.T, np.eye(40), atol=1e-12)


def test_top_db_floor():
    """ScalingTests.swift:113: everything lies within top_db of the max."""
    rng = np.random.default_rng(0)
    S = rng.random(1000) ** 8
    d = O.power_to_db(S, top_db=30.0)
    assert d.min() >= d.max() - 30.0 - 1e-9


# ---------------------------------------------------------------------------
# widening of the path: onset strength, delta, stack_memory, iSTFT
# ---------------------------------------------------------------------------

def test_onset_strength_golden():
    """test_onset_strength.py: librosa.onset.onset_strength(y, sr) defaults."""
    exp = golden("onset_strength_440hz_default")
    got = O.onset_strength(signal_440(), SR)
    assert got.shape == (1, exp.shape[0])
    np.testing.assert_allclose(got[0], exp, rtol=1e-4, atol=1e-4)


def test_delta_and_stack_memory_goldens():
    """test_parity_delta.py (delta atol/rtol 0.1, delta-delta 0.2, stack 1e-4);
    held here to 1e-4 absolute."""
    m = golden("mfcc")
    np.testing.assert_allclose(O.delta(m), golden("delta"), atol=1e-4, rtol=1e-4)
    np.testing.assert_allclose(O.delta(m, order=2), golden("delta_delta"), atol=1e-4, rtol=1e-4)
    np.testing.assert_allclose(O.stack_memory(m, n_steps=3), golden("stack_memory"), atol=1e-6)


def test_istft_inverts_the_oracle_stft():
    """test_parity_istft.py's round trips, as properties: the inverse of the
    forward transform reconstructs the signal (COLA window-sum division)."""
    rng = np.random.default_rng(42)
    for n_fft, L in ((2048, 22050), (1024, 8192), (512, 3001)):
        y = rng.standard_normal(L)
        S = O.stft_complex(y, n_fft, n_fft // 4, n_fft, True)
        r = O.istft(S, n_fft // 4, center=True, length=L)
        np.testing.assert_allclose(r, y, atol=1e-9)
        r2 = O.istft(S, n_fft // 4, center=True)
        assert len(r2) == (S.shape[1] - 1) * (n_fft // 4)


def test_mel_project_and_dct_ortho_goldens():
    """The S= paths (feature.py:50-57, 130-134): the filterbank applied to the
    power spectrogram gives the mel golden, and the DCT-II ortho of its
    power_to_db the MFCC golden; the DCT restatement equals scipy's."""
    from scipy.fftpack import dct
    y = signal_440()
    P = O.stft_power(y, 2048, 512, 2048, True)
    mel = O.mel_project(P, SR, 2048, 128)
    np.testing.assert_allclose(mel, golden("mel_spectrogram_440hz_default"), rtol=1e-4, atol=1e-4)
    C = O.dct_ortho(O.power_to_db(mel), 20)
    np.testing.assert_allclose(C, golden("mfcc_440hz_default"), rtol=1e-4, atol=1e-4)
    S = np.random.default_rng(3).standard_normal((40, 9))
    for n in (13, 40, 60):
        np.testing.assert_allclose(O.dct_ortho(S, n), dct(S, axis=0, type=2, norm="ortho")[:n], atol=1e-12)
