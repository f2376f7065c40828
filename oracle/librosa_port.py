"""NumPy/SciPy restatement of librosa's MFCC pipeline (TEST INFRASTRUCTURE ONLY).

The CPU baseline that stands in for librosa, MetalMom's parity oracle and the
library its benchmark harness times beside it
(``scripts/generate_golden.py:10-81``, ``benchmarks/run_benchmarks.py:19-33``).
librosa is a third-party dependency that is not vendored in the reference
(``pyproject.toml`` dev dependencies, librosa >= 0.11) and is not installed
here, so this module restates its published algorithm for
``librosa.feature.mfcc(y, sr, n_mfcc, n_fft, hop_length, n_mels)``:

    stft: centre padding by n_fft // 2 ("constant", librosa >= 0.10's default),
          frames every hop_length, periodic Hann (scipy ``get_window("hann",
          n_fft, fftbins=True)``), real FFT (pocketfft through ``scipy.fft``)
    melspectrogram: |X|^2 projected on the Slaney-normalised mel filterbank
    power_to_db: 10 log10(max(S, amin) / ref), floored at max - top_db
    mfcc: ``scipy.fft.dct(type=2, norm="ortho", axis=-2)[:n_mfcc]``

in float32 (as librosa keeps a float32 signal's precision), one clip per
worker thread over all host cores.  It is only timed (``bench.py``'s CPU
baseline and reference arm) and checked against the FP64 oracle
(``tests/test_cpu_baselines.py``); the shipped library never calls it.
"""

from __future__ import annotations

import os

import numpy as np
import scipy.fft as sfft

from . import oracle as O


def _window(n_fft: int) -> np.ndarray:
    n = np.arange(n_fft, dtype=np.float64)
    return (0.5 - 0.5 * np.cos(2.0 * np.pi * n / n_fft)).astype(np.float32)


def _frames(y: np.ndarray, n_fft: int, hop: int) -> np.ndarray:
    p = n_fft // 2
    yp = np.pad(np.asarray(y, np.float32), (p, p))
    T = 1 + (len(yp) - n_fft) // hop
    return np.lib.stride_tricks.as_strided(yp, shape=(T, n_fft), strides=(hop * 4, 4), writeable=False)


class Pipeline:
    """One parameter set (sr, n_fft, hop, n_mels, n_mfcc): window and
    filterbank built once, as a caller of librosa that reuses them would."""

    def __init__(self, sr=22050, n_fft=2048, hop=512, n_mels=128, n_mfcc=20, fmin=0.0, fmax=None,
                 top_db=80.0, workers=None):
        self.sr, self.n_fft, self.hop, self.n_mfcc, self.top_db = sr, n_fft, hop, min(n_mfcc, n_mels), top_db
        self.workers = workers or os.cpu_count() or 1
        self.window = _window(n_fft)
        # librosa.filters.mel(norm="slaney", htk=False): the same Slaney bands the
        # oracle builds (pinned there against the reference's filterbank goldens)
        self.fb_t = np.ascontiguousarray(O.mel_filterbank(sr, n_fft, n_mels, fmin, fmax).astype(np.float32).T)

    def mel_db(self, clips):
        """[n_frames, n_mels] float32 log-mel rows of each clip (top_db applied)."""
        frames = [_frames(y, self.n_fft, self.hop) for y in clips]
        stacked = np.concatenate(frames, axis=0) * self.window
        X = sfft.rfft(stacked, axis=-1, workers=self.workers)
        P = X.real * X.real
        P += X.imag * X.imag
        M = P @ self.fb_t
        np.maximum(M, np.float32(1e-10), out=M)
        np.log10(M, out=M)
        M *= np.float32(10.0)
        out, start = [], 0
        for f in frames:
            d = M[start:start + len(f)]
            start += len(f)
            if self.top_db is not None and self.top_db > 0 and len(d):
                np.maximum(d, d.max() - np.float32(self.top_db), out=d)
            out.append(d)
        return out

    def mfcc(self, clips):
        """[n_mfcc, n_frames] float32 MFCC of each clip."""
        res = []
        for d in self.mel_db(clips):
            c = sfft.dct(d, type=2, norm="ortho", axis=-1, workers=self.workers)[:, :self.n_mfcc]
            res.append(np.ascontiguousarray(c.T))
        return res


def mfcc_batch(clips, sr=22050, n_mfcc=20, n_fft=2048, hop=512, n_mels=128, workers=None):
    """MFCC of every clip, one clip per worker thread (all cores by default;
    NumPy's elementwise loops, pocketfft and BLAS release the GIL), each thread
    single-threaded inside (BLAS limited to one thread, FFT workers=1)."""
    from concurrent.futures import ThreadPoolExecutor
    from threadpoolctl import threadpool_limits
    workers = workers or os.cpu_count() or 1
    p = Pipeline(sr, n_fft, hop, n_mels, n_mfcc, workers=1)
    with threadpool_limits(limits=1, user_api="blas"), ThreadPoolExecutor(workers) as ex:
        return list(ex.map(lambda y: p.mfcc([y])[0], clips))
