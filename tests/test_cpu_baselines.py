"""The two CPU stand-ins the bench times for the reference's CPU path, checked
against the FP64 oracle (they are baselines, so they must compute the same
thing): the float32 C port of the reference's per-clip algorithm
(``oracle/refcpu.c``) and the NumPy/SciPy restatement of librosa
(``oracle/librosa_port.py``)."""

import numpy as np

from metalmom_b200 import synth
from oracle import librosa_port, oracle as O, refcpu


def _clips():
    return [synth.music_clip(n, 22050, seed=s) for s, n in ((1, 3 * 22050), (2, 2 * 22050 + 777), (3, 5000))]


def test_librosa_port_matches_oracle():
    clips = _clips()
    outs = librosa_port.mfcc_batch(clips, workers=2)
    p = librosa_port.Pipeline()
    for y, got in zip(clips, outs):
        exp = O.mfcc(y, 22050, 20, 2048, 512, 2048, 128)
        assert got.shape == exp.shape
        assert O.mfcc_rel_error(got, exp) < 1e-4
        d = p.mel_db([y])[0].T
        e = O.mel_db(y, 22050, 2048, 512, 2048, True, 128)
        near = e >= e.max() - 60.0
        assert np.abs(d - e)[near].max() < 1e-3


def test_refcpu_matches_oracle():
    clips = _clips()
    outs = refcpu.mfcc_batch(clips, n_threads=2)
    for y, got in zip(clips, outs):
        exp = O.mfcc(y, 22050, 20, 2048, 512, 2048, 128)
        assert got.shape == exp.shape
        assert O.mfcc_rel_error(got, exp) < 1e-4
        _, d = refcpu.mfcc(y, want_mel_db=True)
        e = O.mel_db(y, 22050, 2048, 512, 2048, True, 128)
        near = e >= e.max() - 60.0
        assert np.abs(d - e)[near].max() < 1e-3


def test_steady_allocator_applies():
    """The bench times the CPU ports with glibc malloc at its steady state
    (large blocks from the heap, freed memory kept); the setting takes on
    this C library."""
    import bench
    assert bench.steady_allocator() is True
