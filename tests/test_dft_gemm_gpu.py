"""DFT as a GEMM on the tensor cores (tcgen05): the precision-comparison
forms of the front end, against the FP64 oracle.

Tolerances (stated per form):
  * BF16x3 (hi*hi + hi*lo + lo*hi, float32 accumulation): MFCC within 1e-4 of
    max |c| (the FP32 bar); mel-dB within 2e-2 dB -- the split keeps about 16
    mantissa bits, and the measured maxima (3e-3 to 8e-3 dB, in bands near the
    top_db floor) are above the 1e-3 dB bar that the FP32 FFT path meets;
  * plain BF16 (reported only, 8-bit mantissas): MFCC within 1e-2 of max |c|,
    mel-dB within 5 dB (measured maxima 1.8 to 2.7 dB);
  * FP16x3 (each frame scaled by a power of two into (-1, 1), fp16 parts
    hi*hi + hi*lo + lo*hi, float32 accumulation): the FP32 bars, MFCC within
    1e-4 of max |c| and mel-dB within 1e-3 dB, also on clips 80 dB quieter
    and louder than full scale;
  * frame counts and shapes exact, as for the FFT path.
"""

import numpy as np
import pytest

import metalmom_b200 as M
from metalmom_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPEECH = dict(sr=16000, n_fft=512, hop_length=160, win_length=400, n_mels=80, n_mfcc=13, fmin=20.0, fmax=8000.0)
TOL = {"bf16x3": (1e-4, 2e-2), "bf16": (1e-2, 5.0), "f16x3": (1e-4, 1e-3)}


def _oracle_mfcc(y, p, pad_mode=O.PAD_CONSTANT):
    return O.mfcc(y, p["sr"], p["n_mfcc"], p["n_fft"], p["hop_length"], p.get("win_length", p["n_fft"]),
                  p["n_mels"], p.get("fmin", 0.0), p.get("fmax"), pad_mode=pad_mode)


@pytest.mark.parametrize("dft", ["bf16x3", "bf16", "f16x3"])
def test_speech_front_end_vs_oracle(dft):
    clips = [synth.speech_clip(L, 16000, seed=L) for L in (1, 255, 257, 3000, 16000, 40001, 160000)]
    outs = M.mfcc_batch(clips, dft=dft, **SPEECH)
    for c, o in zip(clips, outs):
        exp = _oracle_mfcc(c, SPEECH)
        assert o.shape == exp.shape
        if exp.size:
            assert O.mfcc_rel_error(o, exp) < TOL[dft][0], (len(c), O.mfcc_rel_error(o, exp))


@pytest.mark.parametrize("dft", ["bf16x3", "bf16", "f16x3"])
def test_mel_db_error_vs_oracle(dft):
    """The log-mel intermediate of a plan, after the top_db floor."""
    import torch
    clips = [synth.speech_clip(16000 * 4 + 7 * i, 16000, seed=20 + i) for i in range(3)]
    with M.Plan([len(c) for c in clips], dft=dft, **SPEECH) as plan:
        plan.execute_host(clips)
        frame0 = np.concatenate([[0], np.cumsum(plan.frames)])
        for i, c in enumerate(clips):
            T = plan.frames[i]
            ptr = plan.device_mel_db + 4 * int(frame0[i]) * SPEECH["n_mels"]
            mel = torch.as_tensor(_Dev(ptr, T * SPEECH["n_mels"]), device="cuda").cpu().numpy()
            mel = np.maximum(mel.reshape(T, -1).T.astype(np.float64), plan.clip_max_db(i) - 80.0)
            exp = O.mel_db(c, 16000, 512, 160, 400, True, 80, 20.0, 8000.0)
            assert np.abs(mel - exp).max() < TOL[dft][1], np.abs(mel - exp).max()


class _Dev:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 2}


@pytest.mark.parametrize("n_fft,win,hop,pad_mode", [
    (256, 256, 64, "constant"),
    (512, 512, 128, "reflect"),
    (1024, 1024, 256, "constant"),
    (1024, 600, 200, "reflect"),   # window shorter than n_fft, odd support offset
    (512, 401, 160, "constant"),   # odd window lengths
    (1024, 1023, 256, "reflect"),
    (256, 2, 64, "constant"),      # a two-sample window: one K chunk
])
@pytest.mark.parametrize("dft", ["bf16x3", "f16x3"])
def test_sizes_and_padding(n_fft, win, hop, pad_mode, dft):
    p = dict(sr=22050, n_fft=n_fft, hop_length=hop, win_length=win, n_mels=64, n_mfcc=20)
    clips = [synth.music_clip(L, 22050, seed=L + n_fft) for L in (n_fft // 2 + 1, 5 * n_fft + 3, 30001)]
    outs = M.mfcc_batch(clips, dft=dft, pad_mode=pad_mode, **p)
    pm = O.PAD_REFLECT if pad_mode == "reflect" else O.PAD_CONSTANT
    for c, o in zip(clips, outs):
        exp = _oracle_mfcc(c, p, pm)
        assert o.shape == exp.shape
        assert O.mfcc_rel_error(o, exp) < 1e-4, (len(c), O.mfcc_rel_error(o, exp))


def test_many_tiles_batch_equals_single_calls():
    """Tiles of 128 frames across clip boundaries: each clip equals its own call."""
    rng = np.random.default_rng(3)
    clips = [synth.speech_clip(int(L), 16000, seed=i) for i, L in enumerate(rng.integers(100, 60000, 20))]
    outs = M.mfcc_batch(clips, dft="bf16x3", **SPEECH)
    for c, o in zip(clips, outs):
        np.testing.assert_array_equal(o, M.mfcc_batch([c], dft="bf16x3", **SPEECH)[0])


@pytest.mark.parametrize("gain", [1e-4, 1.0, 1e4])
def test_f16x3_frame_scaling_vs_oracle(gain):
    """The fp16 form scales each frame into (-1, 1) before the split: clips 80
    dB quieter or louder than full scale meet the same bars, and a clip with a
    silent stretch (frames of zeros) keeps its floor."""
    y = synth.speech_clip(16000 * 3, 16000, seed=11) * np.float32(gain)
    y[16000:20000] = 0.0
    out = M.mfcc_batch([y], dft="f16x3", **SPEECH)[0]
    assert O.mfcc_rel_error(out, _oracle_mfcc(y, SPEECH)) < 1e-4
    with M.Plan([len(y)], dft="f16x3", **SPEECH) as plan:
        plan.execute_host([y])
        T = plan.frames[0]
        mel = torch_rows(plan.clip_mel_db_ptr(0), T * SPEECH["n_mels"])
        mel = np.maximum(mel.reshape(T, -1).T.astype(np.float64), plan.clip_max_db(0) - 80.0)
        exp = O.mel_db(y, 16000, 512, 160, 400, True, 80, 20.0, 8000.0)
        assert np.abs(mel - exp).max() < 1e-3, np.abs(mel - exp).max()


def torch_rows(ptr, n):
    import torch
    return torch.as_tensor(_Dev(ptr, n), device="cuda").cpu().numpy()


@pytest.mark.parametrize("dft", ["bf16x3", "f16x3"])
def test_non_finite_input_and_unsupported_sizes(dft):
    y = synth.speech_clip(8000, 16000, seed=1)
    y[3000] = np.nan
    o = M.mfcc_batch([y], dft=dft, **SPEECH)[0]
    assert o.shape == (13, 51)
    with pytest.raises(RuntimeError, match="status -1"):
        M.mfcc_batch([y], dft="bf16x3", sr=22050, n_fft=2048)  # the GEMM forms stop at n_fft 1024

