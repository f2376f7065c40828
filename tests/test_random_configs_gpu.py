"""Seeded random front-end configurations against the FP64 oracle.

Each case draws a sample rate, n_fft (16..4096), hop, window length,
band count, fmin / fmax, MFCC count, clip length and padding, and checks
mm_mfcc (MFCC within 1e-4 of max |c|) and mm_mel_spectrogram through the C
ABI, and the batched entry point with the clip in a mixed batch (bitwise
equal to the single call).

Mel-dB tolerance (``dbcheck.check_db``): 1e-3 dB for values within 60 dB of
the clip's maximum; 60-70 and 70-80 dB below it, no worse than FACTOR times
the error of the reference's own float32 path (``oracle/refcpu.c``) on the
same draw and distance bin, or 1e-3 dB when that is larger.  The float32
FFT's rounding is absolute (a fraction of the frame's largest bins), so its dB
error grows with the distance below the maximum, in the reference's float32
path as on the GPU.

The draw covers the kernel choices the library makes on its own (the warp
kernels for n_fft 2048 and 4096, the CTA-tile kernels of every size, the tiny
direct-DFT kernel), and each draw runs again with the warp kernels forced for
n_fft 256..4096 (lane tables or packed rows); sizes and modes without them
keep their own kernel.
"""

import numpy as np
import pytest

import metalmom_b200 as M
from dbcheck import check_db
from metalmom_b200 import synth
from oracle import oracle as O, refcpu

pytestmark = pytest.mark.gpu

MFCC_TOL = 1e-4


def _draw(seed):
    rng = np.random.default_rng(seed)
    sr = int(rng.choice([8000, 16000, 22050, 44100]))
    n_fft = int(2 ** rng.integers(4, 13))
    hop = int(max(1, n_fft // int(rng.choice([1, 2, 3, 4, 8]))))
    win = int(rng.integers(max(1, n_fft // 4), n_fft + 1)) if rng.random() < 0.4 else n_fft
    n_mels = int(rng.integers(1, min(160, 8 + n_fft // 8)))
    fmin = float(rng.choice([0.0, 20.0, 100.0, 300.0]))
    fmax = None if rng.random() < 0.5 else float(rng.uniform(fmin + 500.0, sr / 2.0))
    n_mfcc = int(rng.integers(1, 40))
    L = int(rng.integers(1, 4 * sr))
    pad = "reflect" if (rng.random() < 0.25 and L > n_fft // 2) else "constant"
    return dict(sr=sr, n_fft=n_fft, hop=hop, win=win, n_mels=n_mels, fmin=fmin, fmax=fmax, n_mfcc=n_mfcc, L=L,
                pad=pad)


@pytest.fixture(params=[None, 3], ids=["default", "warp"])
def variant(request):
    """The library's own kernel choice, then the warp kernels (launch variant
    3, n_fft 256..4096) forced for every size that has them."""
    if request.param is None:
        yield None
        return
    sizes = [1 << b for b in range(4, 16)]
    old = {n: M.tune_get(n) for n in sizes}
    for n in sizes:
        M.tune_set(n, request.param)
    try:
        yield request.param
    finally:
        for n, v in old.items():
            M.tune_set(n, v)


@pytest.mark.parametrize("seed", range(40))
def test_random_config_vs_oracle(seed, variant):
    c = _draw(seed)
    y = synth.music_clip(c["L"], c["sr"], seed=seed)
    pm = O.PAD_REFLECT if c["pad"] == "reflect" else O.PAD_CONSTANT
    kw = dict(sr=c["sr"], n_fft=c["n_fft"], hop_length=c["hop"], win_length=c["win"], n_mels=c["n_mels"],
              fmin=c["fmin"], fmax=c["fmax"])
    exp = O.mfcc(y, c["sr"], c["n_mfcc"], c["n_fft"], c["hop"], c["win"], c["n_mels"], c["fmin"], c["fmax"], True,
                 pad_mode=pm)
    if c["pad"] == "constant":  # the reference's per-clip entry points pad with zeros only
        got = M.mfcc(y, n_mfcc=c["n_mfcc"], **kw)
        assert got.shape == exp.shape, c
        if exp.size:
            assert O.mfcc_rel_error(got, exp) < MFCC_TOL, (c, O.mfcc_rel_error(got, exp))
        mel = M.melspectrogram(y, **kw)
        got_db = O.power_to_db(np.asarray(mel, np.float64), 1.0, 1e-10, 80.0)
        exp_db = O.mel_db(y, c["sr"], c["n_fft"], c["hop"], c["win"], True, c["n_mels"], c["fmin"], c["fmax"])
        if exp_db.size:
            _, ref_db = refcpu.mfcc(y, c["sr"], c["n_mfcc"], c["n_fft"], c["hop"], c["win"], c["n_mels"], c["fmin"],
                                    c["fmax"] or 0.0, True, want_mel_db=True)
            check_db(got_db, exp_db, ref_db, c)
    # batched, with the padding mode of the draw, next to a clip of another length
    other = synth.music_clip(c["L"] // 3 + 7, c["sr"], seed=seed + 1000)
    bkw = dict(kw, n_mfcc=c["n_mfcc"], pad_mode=c["pad"])
    outs = M.mfcc_batch([other, y], **bkw)
    assert outs[1].shape == exp.shape, c
    if exp.size:
        assert O.mfcc_rel_error(outs[1], exp) < MFCC_TOL, (c, O.mfcc_rel_error(outs[1], exp))
    np.testing.assert_array_equal(outs[1], M.mfcc_batch([y], **bkw)[0])
