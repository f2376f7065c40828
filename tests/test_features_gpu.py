"""Features built on the front end, through the C ABI, against the reference's
goldens and the FP64 oracle.

Tolerances: onset strength -- the reference's test tolerance (rtol=atol=1e-4)
against its librosa golden and 1e-3 of the envelope maximum against the
oracle (float32 mel dB differences); delta / stack_memory -- 1e-4 absolute
(the reference's own tests allow 0.1 / 0.2 for delta, 1e-4 for stack_memory).
"""

import numpy as np
import pytest

import metalmom_b200 as M
from metalmom_b200 import synth
from goldens import golden, signal_440
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_onset_strength_golden():
    exp = golden("onset_strength_440hz_default")
    got = M.onset_strength(y=signal_440(), sr=22050)
    assert got.shape == exp.shape
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("n_fft,hop,n_mels,center,L", [
    (2048, 512, 128, True, 661500),
    (1024, 256, 64, True, 44100),
    (2048, 512, 40, False, 30000),
    (512, 128, 32, True, 7000),
    (2048, 0, 128, True, 22050),    # hop sentinel -> 512
])
def test_onset_strength_vs_oracle(n_fft, hop, n_mels, center, L):
    y = synth.music_clip(L, 22050, seed=L + n_fft)
    h = hop if hop > 0 else 512
    for aggregate in (True, False):
        got = M.onset_strength(y=y, sr=22050, n_fft=n_fft, hop_length=hop, n_mels=n_mels,
                               center=center, aggregate=aggregate)
        exp = O.onset_strength(y, 22050, n_fft, h, n_mels, center=center, aggregate=aggregate)
        exp = exp.ravel() if aggregate else exp
        assert got.shape == exp.shape
        assert np.abs(got - exp).max() <= 1e-3 * max(np.abs(exp).max(), 1.0)


def test_onset_strength_short_signals():
    one = M.onset_strength(y=np.ones(100, np.float32), sr=22050, center=False)   # no frame
    assert one.shape == (1,) and one[0] == 0.0
    few = M.onset_strength(y=synth.music_clip(600, 22050, seed=3), sr=22050)     # 2 frames
    np.testing.assert_allclose(few, O.onset_strength(synth.music_clip(600, 22050, seed=3), 22050).ravel(),
                               atol=1e-4)
    with pytest.raises(RuntimeError, match="status -1"):
        M.onset_strength(y=np.ones(4096, np.float32), n_mels=0)


def test_delta_goldens():
    m = golden("mfcc")
    np.testing.assert_allclose(M.delta(m), golden("delta"), atol=1e-4, rtol=1e-4)
    np.testing.assert_allclose(M.delta(m, order=2), golden("delta_delta"), atol=1e-4, rtol=1e-4)
    np.testing.assert_allclose(M.stack_memory(m, n_steps=3), golden("stack_memory"), atol=1e-6)


@pytest.mark.parametrize("width,order", [(3, 1), (5, 2), (9, 1), (9, 3), (21, 2)])
def test_delta_vs_oracle(width, order):
    rng = np.random.default_rng(width * 10 + order)
    x = rng.standard_normal((13, 77)).astype(np.float32)
    got = M.delta(x, width=width, order=order)
    exp = O.delta(x, width, order)
    assert np.abs(got - exp).max() <= 1e-4 * max(np.abs(exp).max(), 1.0)
    assert np.abs(M.delta(np.full((4, 20), 5.0, np.float32))).max() < 1e-5


def test_delta_and_stack_memory_edges():
    x = np.arange(60, dtype=np.float32).reshape(3, 20)
    for n_steps, delay in ((1, 1), (3, 2), (2, 25), (2, -1)):
        np.testing.assert_array_equal(M.stack_memory(x, n_steps=n_steps, delay=delay),
                                      O.stack_memory(x, n_steps, delay).astype(np.float32))
    with pytest.raises(RuntimeError, match="status -1"):
        M.delta(np.ones((2, 5), np.float32), width=9)   # fewer frames than the window
    with pytest.raises(RuntimeError, match="status -1"):
        M.delta(np.ones((2, 50), np.float32), width=4)  # even width
