"""The tensor-core frame kernel (launch variant 5, n_fft 2048, MFCC path):
both 32-point DFT stages as fp16x3 tcgen05 GEMMs with each frame scaled by a
power of two.  Checked against the FP64 oracle at the FP32 bars (MFCC within
1e-4 of max |c|; mel-dB within 1e-3 dB within 60 dB of the clip maximum and
bounded by the reference's float32 path below that), on clips of every length
class (edge frames, one frame, odd offsets in a batch), quiet and loud
clips, non-finite and ~1e17 samples, the packed-row filterbank epilogue, and
bitwise batch/single equality."""

import numpy as np
import pytest

import metalmom_b200 as M
from dbcheck import check_db
from metalmom_b200 import synth
from oracle import oracle as O, refcpu

pytestmark = pytest.mark.gpu

SR = 22050
MFCC_TOL = 1e-4


@pytest.fixture
def tc():
    old = M.tune_get(2048)
    M.tune_set(2048, 5)
    try:
        yield
    finally:
        M.tune_set(2048, old)


def _device_floats(ptr, n):
    import torch

    class View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 2}

    return torch.as_tensor(View(), device="cuda").cpu().numpy().copy()


@pytest.mark.parametrize("L", [1, 1023, 1024, 2049, 5 * SR + 333, 30 * SR])
def test_tc_kernel_mfcc_vs_oracle(tc, L):
    y = synth.music_clip(L, SR, seed=L)
    got = M.mfcc(y, sr=SR)
    exp = O.mfcc(y, SR, 20, 2048, 512, 2048, 128)
    assert got.shape == exp.shape
    if exp.size:
        assert O.mfcc_rel_error(got, exp) < MFCC_TOL, O.mfcc_rel_error(got, exp)


@pytest.mark.parametrize("gain", [1e-6, 1.0, 1e6])
def test_tc_kernel_mel_db_vs_oracle_and_reference_path(tc, gain):
    """The plan's log-mel rows (after the floor) at three signal levels: the
    per-frame scale keeps the fp16 split at float32 grade whatever the level."""
    clips = [synth.music_clip(10 * SR + 77 * i, SR, seed=40 + i) * np.float32(gain) for i in range(3)]
    clips[1][SR:2 * SR] = 0.0  # a silent second: frames of zeros
    with M.Plan([len(c) for c in clips], sr=SR, n_fft=2048, hop_length=512, n_mels=128, n_mfcc=20) as plan:
        outs = plan.execute_host(clips)
        for i, y in enumerate(clips):
            T = plan.frames[i]
            rows = _device_floats(plan.clip_mel_db_ptr(i), T * 128).reshape(T, 128).T
            got_db = np.maximum(rows.astype(np.float64), plan.clip_max_db(i) - 80.0)
            exp_db = O.mel_db(y, SR, 2048, 512, 2048, True, 128)
            _, ref_db = refcpu.mfcc(y, SR, 20, 2048, 512, 2048, 128, 0.0, 0.0, True, want_mel_db=True)
            check_db(got_db, exp_db, ref_db, (gain, i))
            assert O.mfcc_rel_error(outs[i], O.dct_basis(20, 128) @ exp_db) < MFCC_TOL


def test_tc_kernel_close_to_warp_kernel_and_batch_equals_single(tc):
    lens = [700, 3 * SR + 1, SR // 2, 7 * SR + 13, 2048 * 3]
    clips = [synth.music_clip(L, SR, seed=90 + i) for i, L in enumerate(lens)]
    outs = M.mfcc_batch(clips, sr=SR)
    for c, o in zip(clips, outs):
        np.testing.assert_array_equal(o, M.mfcc_batch([c], sr=SR)[0])
    M.tune_set(2048, 3)
    warp = M.mfcc_batch(clips, sr=SR)
    for o, w in zip(outs, warp):
        assert o.shape == w.shape
        assert np.abs(o - w).max() <= 1e-4 * np.abs(w).max()


def test_tc_kernel_non_finite_and_large_samples(tc):
    y = synth.music_clip(3 * SR, SR, seed=37)
    y[9000] = np.nan
    y[40000] = np.inf
    got = M.mfcc(y, sr=SR)
    with np.errstate(all="ignore"):
        exp = O.mfcc(y, SR, 20, 2048, 512, 2048, 128)
    assert got.shape == exp.shape and np.isfinite(got).all()
    assert O.mfcc_rel_error(got, exp) < MFCC_TOL
    rng = np.random.default_rng(11)
    big = (rng.standard_normal(2 * SR) * 1e17).astype(np.float32)
    assert O.mfcc_rel_error(M.mfcc(big, sr=SR), O.mfcc(big, SR, 20, 2048, 512, 2048, 128)) < MFCC_TOL


@pytest.mark.parametrize("n_mels,fmin,fmax", [(40, 0.0, None), (256, 20.0, 8000.0), (1100, 0.0, None)])
def test_tc_kernel_filterbank_shapes(tc, n_mels, fmin, fmax):
    """Lane tables (40, 256 bands) and the packed-row epilogue (1100 bands)."""
    y = synth.music_clip(4 * SR, SR, seed=n_mels)
    got = M.mfcc(y, sr=SR, n_mfcc=32, n_mels=n_mels, fmin=fmin, fmax=fmax)
    with np.errstate(all="ignore"):
        exp = O.mfcc(y, SR, 32, 2048, 512, 2048, n_mels, fmin, fmax)
    assert got.shape == exp.shape
    assert O.mfcc_rel_error(got, exp) < MFCC_TOL, O.mfcc_rel_error(got, exp)
