"""CPU oracle for the spectral front end (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The shipped library
(``metalmom_b200/_lib/libmetalmom.so``) never calls into it.

It restates MetalMom's CPU algorithm for the path

    centered framing -> periodic Hann -> real FFT -> |X|^2 -> Slaney mel
    -> power_to_db(top_db) -> DCT-II ortho (MFCC)

and for the features built on it (onset strength, inverse STFT, delta,
stack_memory) in float64 NumPy.  Each function cites the Swift source it follows (paths
relative to the MetalMom project root).  The FFT itself is ``numpy.fft.rfft``
in float64: the reference calls Apple's closed ``vDSP_fft_zrip`` and rescales by
0.5 so that its output is the plain DFT (``STFT.swift:298-310``); any exact
float64 DFT is therefore a faithful stand-in.

Pinning: ``tests/test_oracle_golden.py`` checks this module against the
reference's own librosa-generated golden vectors (``Tests/golden/*.npy``,
copied into ``tests/golden/reference_goldens.npz`` by
``tests/golden/make_golden.py``) at the reference's tolerances.

Padding: the reference (and its goldens) pad with ZEROS when ``center`` is set
(``STFT.swift:241-249``).  ``pad_mode="reflect"`` is an additional mode
(librosa's older default); ``"constant"`` is the default everywhere.
"""

from __future__ import annotations

import math

import numpy as np

PAD_CONSTANT = "constant"
PAD_REFLECT = "reflect"


# ---------------------------------------------------------------------------
# Framing (STFT.swift:241-254, executeCPU :81-98)
# ---------------------------------------------------------------------------

def is_power_of_two(n: int) -> bool:
    """``isPowerOfTwo`` (STFT.swift:34-37)."""
    return n > 0 and (n & (n - 1)) == 0


def n_frames(length: int, n_fft: int, hop: int, center: bool) -> int:
    """Frame count exactly as ``STFT.computePowerSpectrogram`` computes it.

    ``padded = L + 2*(n_fft/2)`` when centered (STFT.swift:241-249); zero frames
    when ``padded < n_fft`` (:251-253); otherwise ``1 + (padded-n_fft)/hop``
    with integer (floor) division (:254).  A non-power-of-two ``n_fft`` also
    yields zero frames (:260-262).
    """
    padded = length + 2 * (n_fft // 2) if center else length
    if padded < n_fft:
        return 0
    if not is_power_of_two(n_fft):
        return 0
    return 1 + (padded - n_fft) // hop


def pad_signal(y: np.ndarray, n_fft: int, center: bool,
               pad_mode: str = PAD_CONSTANT) -> np.ndarray:
    """Center padding by ``n_fft//2`` on both sides (STFT.swift:241-249).

    ``constant`` pads zeros (the reference); ``reflect`` mirrors without
    repeating the edge sample, folding repeatedly for very short signals.
    """
    y = np.asarray(y, dtype=np.float64)
    if not center:
        return y
    p = n_fft // 2
    if pad_mode == PAD_CONSTANT:
        return np.concatenate([np.zeros(p), y, np.zeros(p)])
    if pad_mode == PAD_REFLECT:
        idx = np.arange(-p, len(y) + p)
        return y[reflect_index(idx, len(y))]
    raise ValueError(f"unknown pad_mode {pad_mode!r}")


def reflect_index(idx: np.ndarray, length: int) -> np.ndarray:
    """Fold integer indices into [0, length) by mirror reflection (no edge repeat)."""
    idx = np.asarray(idx, dtype=np.int64)
    if length <= 1:
        return np.zeros_like(idx)
    period = 2 * (length - 1)
    m = np.mod(idx, period)
    return np.where(m < length, m, period - m)


# ---------------------------------------------------------------------------
# Window (Windows.swift:14-48, prepareWindow STFT.swift:44-57)
# ---------------------------------------------------------------------------

def hann_periodic(length: int) -> np.ndarray:
    """Periodic Hann ``0.5 - 0.5 cos(2 pi n / length)`` (Windows.swift:14-48).

    Length <= 0 gives an empty window and length 1 gives ``[1.0]``
    (Windows.swift:15-16).
    """
    if length <= 0:
        return np.zeros(0)
    if length == 1:
        return np.ones(1)
    n = np.arange(length, dtype=np.float64)
    return 0.5 - 0.5 * np.cos(2.0 * np.pi * n / length)


def prepare_window(win_length: int, n_fft: int) -> np.ndarray:
    """Full-length analysis window of exactly ``n_fft`` samples (STFT.swift:44-57).

    Shorter windows are zero-padded with ``(n_fft-win)//2`` zeros in front;
    longer windows keep their centre ``n_fft`` samples.  A window length
    <= 0 (reachable only through ``mm_stft``, which applies no sentinel) gives
    an all-zero window, as the reference's empty Hann does.
    """
    if win_length <= 0:
        return np.zeros(n_fft)
    w = hann_periodic(win_length)
    if win_length < n_fft:
        before = (n_fft - win_length) // 2
        after = n_fft - win_length - before
        return np.concatenate([np.zeros(before), w, np.zeros(after)])
    if win_length > n_fft:
        start = (win_length - n_fft) // 2
        return w[start:start + n_fft]
    return w


# ---------------------------------------------------------------------------
# STFT power / magnitude (STFT.swift:227-340, executeCPU :73-215)
# ---------------------------------------------------------------------------

def frames_matrix(y, n_fft, hop, win_length, center, pad_mode=PAD_CONSTANT):
    """Windowed frames [n_frames, n_fft] in float64 (STFT.swift:287-296)."""
    nfr = n_frames(len(y), n_fft, hop, center)
    if nfr == 0:
        return np.zeros((0, n_fft))
    yp = pad_signal(y, n_fft, center, pad_mode)
    w = prepare_window(win_length, n_fft)
    starts = np.arange(nfr, dtype=np.int64) * hop
    idx = starts[:, None] + np.arange(n_fft, dtype=np.int64)[None, :]
    return yp[idx] * w[None, :]


def stft_complex(y, n_fft, hop, win_length, center, pad_mode=PAD_CONSTANT):
    """Complex DFT of every windowed frame, shape [n_fft//2+1, n_frames]."""
    fr = frames_matrix(y, n_fft, hop, win_length, center, pad_mode)
    nfreq = n_fft // 2 + 1
    if fr.shape[0] == 0:
        return np.zeros((nfreq, 0), dtype=np.complex128)
    return np.fft.rfft(fr, axis=1).T


def stft_power(y, n_fft, hop, win_length, center, pad_mode=PAD_CONSTANT):
    """``|X|^2`` in layout [n_freqs, n_frames] (STFT.swift:312-335)."""
    X = stft_complex(y, n_fft, hop, win_length, center, pad_mode)
    return X.real ** 2 + X.imag ** 2


def stft_magnitude(y, n_fft, hop, win_length, center, pad_mode=PAD_CONSTANT):
    """``|X|`` in layout [n_freqs, n_frames] (executeCPU, STFT.swift:170-197)."""
    return np.sqrt(stft_power(y, n_fft, hop, win_length, center, pad_mode))


# ---------------------------------------------------------------------------
# Slaney mel filterbank (FilterBank.swift:23-73, Units.swift:55-85)
# ---------------------------------------------------------------------------

_F_SP = 200.0 / 3.0
_MIN_LOG_HZ = 1000.0
_MIN_LOG_MEL = _MIN_LOG_HZ / _F_SP
_LOGSTEP = math.log(6.4) / 27.0


def hz_to_mel(hz: float) -> float:
    """Slaney Hz -> mel in float64 (``Units.hzToMelD``, Units.swift:55-67)."""
    mel = hz / _F_SP
    if hz >= _MIN_LOG_HZ:
        mel = _MIN_LOG_MEL + math.log(hz / _MIN_LOG_HZ) / _LOGSTEP
    return mel


def mel_to_hz(mel: float) -> float:
    """Slaney mel -> Hz in float64 (``Units.melToHzD``, Units.swift:74-85)."""
    if mel < _MIN_LOG_MEL:
        return mel * _F_SP
    return _MIN_LOG_HZ * math.exp((mel - _MIN_LOG_MEL) * _LOGSTEP)


def mel_points(sr: int, n_mels: int, fmin: float, fmax: float) -> np.ndarray:
    """``n_mels+2`` band edges in Hz, float64 (FilterBank.swift:33-40)."""
    lo = hz_to_mel(float(fmin))
    hi = hz_to_mel(float(fmax))
    return np.array([mel_to_hz(lo + i * (hi - lo) / (n_mels + 1))
                     for i in range(n_mels + 2)], dtype=np.float64)


def mel_filterbank(sr: int, n_fft: int, n_mels: int = 128, fmin: float = 0.0,
                   fmax: float | None = None) -> np.ndarray:
    """Slaney-normalised triangular filterbank [n_mels, n_fft//2+1] in float64.

    Same tests and ordering as FilterBank.swift:51-70: a bin belongs to the
    rising edge when ``left <= f <= centre`` (and ``centre != left``), to the
    falling edge when ``centre < f <= right`` (and ``right != centre``); each
    row is then scaled by ``2/(right-left)`` (which turns a degenerate row
    into NaN, as the reference's ``0 * inf`` does).
    """
    if fmax is None or fmax <= 0:
        fmax = sr / 2.0
    nfreq = n_fft // 2 + 1
    pts = mel_points(sr, n_mels, fmin, fmax)
    freqs = np.arange(nfreq, dtype=np.float64) * sr / n_fft
    W = np.zeros((n_mels, nfreq))
    with np.errstate(divide="ignore", invalid="ignore"):
        for m in range(n_mels):
            fl, fc, fr = pts[m], pts[m + 1], pts[m + 2]
            rise = (freqs >= fl) & (freqs <= fc) & (fc != fl)
            fall = (~rise) & (freqs > fc) & (freqs <= fr) & (fr != fc)
            if fc != fl:
                W[m, rise] = (freqs[rise] - fl) / (fc - fl)
            if fr != fc:
                W[m, fall] = (fr - freqs[fall]) / (fr - fc)
            W[m, :] *= 2.0 / (fr - fl) if fr != fl else np.inf
    return W


# ---------------------------------------------------------------------------
# dB scaling (Scaling.swift:39-42, 73-118)
# ---------------------------------------------------------------------------

def _vthr(x: np.ndarray, t) -> np.ndarray:
    """vDSP_vthr as documented: ``x if x >= t else t`` (NaN -> t)."""
    return np.where(x >= t, x, t)


def linear_to_db(S, multiplier: float, ref: float = 1.0, amin: float = 1e-10,
                 top_db: float | None = 80.0) -> np.ndarray:
    """``multiplier*log10(max(S, amin)/ref)`` then the top_db floor.

    The floor is ``max(result) - top_db`` over the WHOLE array
    (Scaling.swift:106-114); ``top_db`` None (or <= 0 at the C ABI,
    Bridge.swift:286) disables it.
    """
    S = np.asarray(S, dtype=np.float64)
    if S.size == 0:
        return S.copy()
    with np.errstate(divide="ignore", invalid="ignore"):
        out = multiplier * np.log10(_vthr(S, amin) / ref)
    if top_db is not None and top_db > 0:
        finite = out[~np.isnan(out)]
        vmax = finite.max() if finite.size else np.nan
        out = _vthr(out, vmax - top_db)
    return out


def power_to_db(S, ref=1.0, amin=1e-10, top_db=80.0):
    """``Scaling.powerToDb`` (Scaling.swift:39-42)."""
    return linear_to_db(S, 10.0, ref, amin, top_db)


def amplitude_to_db(S, ref=1.0, amin=1e-5, top_db=80.0):
    """``Scaling.amplitudeToDb`` (Scaling.swift:23-26)."""
    return linear_to_db(S, 20.0, ref, amin, top_db)


# ---------------------------------------------------------------------------
# Mel spectrogram and MFCC (MelSpectrogram.swift:28-142, MFCC.swift:28-110)
# ---------------------------------------------------------------------------

def melspectrogram(y, sr=22050, n_fft=2048, hop=None, win_length=None,
                   center=True, power=2.0, n_mels=128, fmin=0.0, fmax=None,
                   pad_mode=PAD_CONSTANT):
    """``MelSpectrogram.compute``: ``FB @ |X|^power`` [n_mels, n_frames].

    ``hop``/``win_length`` None mean ``n_fft//4`` / ``n_fft``
    (MelSpectrogram.swift via STFT.swift:239-240).
    """
    hop = n_fft // 4 if hop is None else hop
    win = n_fft if win_length is None else win_length
    P = stft_power(y, n_fft, hop, win, center, pad_mode)
    if power != 2.0:
        P = np.sqrt(P) ** power
    FB = mel_filterbank(sr, n_fft, n_mels, fmin, fmax)
    if P.shape[1] == 0:
        return np.zeros((n_mels, 0))
    return FB @ P


def dct_basis(n_mfcc: int, n_mels: int) -> np.ndarray:
    """DCT-II ortho basis [n_mfcc, n_mels] (MFCC.swift:79-88), float64."""
    k = np.arange(n_mfcc, dtype=np.float64)[:, None]
    n = np.arange(n_mels, dtype=np.float64)[None, :]
    B = np.cos(np.pi * k * (2.0 * n + 1.0) / (2.0 * n_mels))
    B[0, :] *= math.sqrt(1.0 / n_mels)
    B[1:, :] *= math.sqrt(2.0 / n_mels)
    return B


def mel_db(y, sr=22050, n_fft=2048, hop=None, win_length=None, center=True,
           n_mels=128, fmin=0.0, fmax=None, top_db=80.0, pad_mode=PAD_CONSTANT):
    """``Scaling.powerToDb(melSpec)`` with ref 1, amin 1e-10 (MFCC.swift:57)."""
    M = melspectrogram(y, sr, n_fft, hop, win_length, center, 2.0, n_mels,
                       fmin, fmax, pad_mode)
    return power_to_db(M, 1.0, 1e-10, top_db)


def mfcc(y, sr=22050, n_mfcc=20, n_fft=2048, hop=None, win_length=None,
         n_mels=128, fmin=0.0, fmax=None, center=True, pad_mode=PAD_CONSTANT,
         top_db=80.0):
    """``MFCC.compute``: DCT-II ortho of the log-mel, first ``min(n_mfcc, n_mels)``
    rows (MFCC.swift:28-110)."""
    D = mel_db(y, sr, n_fft, hop, win_length, center, n_mels, fmin, fmax,
               top_db, pad_mode)
    k = min(n_mfcc, n_mels)
    if D.shape[1] == 0 or k <= 0:
        return np.zeros((max(k, 0), D.shape[1]))
    return dct_basis(k, n_mels) @ D


def mel_project(S, sr=22050, n_fft=2048, n_mels=128, fmin=0.0, fmax=None):
    """``melspectrogram(S=...)``: the Slaney filterbank applied to a given
    [n_freqs, n_frames] spectrogram (python/metalmom/feature.py:50-57, which
    multiplies the ``_mel_fb.py`` filterbank into S), in float64."""
    return mel_filterbank(sr, n_fft, n_mels, fmin, fmax) @ np.asarray(S, np.float64)


def dct_ortho(S, n_out):
    """``mfcc(S=...)``: DCT-II ortho along axis 0 of [n_rows, n_frames], first
    ``n_out`` rows (feature.py:130-134, scipy ``dct(type=2, norm='ortho')``)."""
    S = np.asarray(S, np.float64)
    k = min(n_out, S.shape[0])
    return dct_basis(k, S.shape[0]) @ S


# ---------------------------------------------------------------------------
# Widening of the path: onset strength, iSTFT, delta, stack_memory
# ---------------------------------------------------------------------------

def onset_strength(y, sr=22050, n_fft=2048, hop=None, n_mels=128, fmin=0.0,
                   fmax=None, center=True, aggregate=True, lag=1,
                   pad_mode=PAD_CONSTANT):
    """``OnsetDetection.onsetStrength`` (Rhythm/OnsetDetection.swift:23-139).

    Power mel spectrogram (window n_fft, hop default 512) -> power_to_db(ref
    1, amin 1e-10, top_db 80) -> positive lag difference along time -> mean
    over bands (or per band), shifted right by ``lag + n_fft // (2 hop)``
    when centered (``lag`` otherwise) with zeros in front; ``n_frames``
    columns (``[1, 1]`` / ``[n_mels, 1]`` zeros when there are <= lag frames).
    """
    hop = 512 if hop is None else hop
    S = mel_db(y, sr, n_fft, hop, n_fft, center, n_mels, fmin, fmax, 80.0, pad_mode)
    n_bands, T = S.shape
    if T <= lag:
        return np.zeros((1, 1)) if aggregate else np.zeros((n_bands, 1))
    diff = np.maximum(0.0, S[:, lag:] - S[:, :-lag])
    pad = lag + (n_fft // (2 * hop) if center else 0)
    out_frames = min(diff.shape[1] + pad, T) if center else diff.shape[1] + pad
    full = np.zeros((n_bands, out_frames))
    n = min(diff.shape[1], out_frames - pad)
    if n > 0:
        full[:, pad:pad + n] = diff[:, :n]
    return full.mean(axis=0, keepdims=True) if aggregate else full


def istft(S, hop=None, win_length=None, center=True, length=None):
    """``STFT.inverse`` (Spectral/STFT.swift:686-860): inverse real DFT of
    every frame, synthesis window, overlap-add, division by the overlapped
    squared windows where their sum exceeds 1e-10, then trimming of the
    centre padding / ``length``.  ``S`` is complex [n_freqs, n_frames]; a
    non-power-of-two n_fft gives zeros of the padded length (:719-724)."""
    S = np.asarray(S)
    n_freqs, T = S.shape
    n_fft = (n_freqs - 1) * 2
    hop = n_fft // 4 if hop is None else hop
    win = n_fft if win_length is None else win_length
    expected = n_fft + (T - 1) * hop
    w = prepare_window(win, n_fft)
    if not is_power_of_two(n_fft):
        out = np.zeros(expected)
    else:
        X = S.astype(np.complex128).copy()
        X[0] = X[0].real          # DC and Nyquist: real parts only (:747-753)
        X[-1] = X[-1].real
        frames = np.fft.irfft(X.T, n=n_fft, axis=1) * w[None, :]
        out = np.zeros(expected)
        wsum = np.zeros(expected)
        for f in range(T):
            out[f * hop:f * hop + n_fft] += frames[f]
            wsum[f * hop:f * hop + n_fft] += w * w
        nz = wsum > 1e-10
        out[nz] /= wsum[nz]
    if center:
        a = n_fft // 2
        if length is not None:
            r = out[a:min(a + length, expected)]
            return np.concatenate([r, np.zeros(length - len(r))]) if len(r) < length else r
        b = expected - n_fft // 2
        return out[a:b] if b > a else np.zeros(0)
    if length is not None:
        return out[:length] if len(out) >= length else np.concatenate([out, np.zeros(length - len(out))])
    return out


def savgol_coeffs(width: int, order: int) -> np.ndarray:
    """Savitzky-Golay derivative coefficients (Features/Delta.swift:30-135):
    row ``order`` of pinv(V), V[i, j] = (i - width//2)^j, j <= order, times
    ``order!``; coefficient k multiplies the sample at offset k - width//2."""
    half = width // 2
    x = np.arange(width, dtype=np.float64) - half
    V = np.vander(x, order + 1, increasing=True)
    return np.linalg.pinv(V)[order] * math.factorial(order)


def delta(data, width=9, order=1):
    """``Delta.compute`` (Features/Delta.swift:137-241), librosa's
    ``mode='interp'``: interior frames by the SG filter; the first and last
    ``width//2`` frames take the filter applied to the first / last ``width``
    frames."""
    D = np.asarray(data, dtype=np.float64)
    nf, T = D.shape
    half = width // 2
    c = savgol_coeffs(width, order)
    out = np.zeros_like(D)
    for t in range(half, T - half):
        out[:, t] = D[:, t - half:t + half + 1] @ c
    left = D[:, :width] @ c
    right = D[:, T - width:] @ c
    out[:, :half] = left[:, None]
    out[:, T - half:] = right[:, None]
    return out


def stack_memory(data, n_steps=2, delay=1):
    """``Delta.stackMemory`` (Features/Delta.swift:256-290): rows
    ``step*n_features + f`` hold the features delayed by ``step*delay``
    frames, zeros before the start."""
    D = np.asarray(data, dtype=np.float64)
    nf, T = D.shape
    out = np.zeros((nf * n_steps, T))
    for step in range(n_steps):
        sh = step * delay  # output frame t takes input frame t - sh
        rows = slice(step * nf, (step + 1) * nf)
        if 0 <= sh < T:
            out[rows, sh:] = D[:, :T - sh]
        elif -T < sh < 0:
            out[rows, :T + sh] = D[:, -sh:]
    return out


# ---------------------------------------------------------------------------
# Error metrics used by the parity tests and the bench
# ---------------------------------------------------------------------------

def mel_db_error(test_db: np.ndarray, oracle_db: np.ndarray) -> tuple[float, float]:
    """(max, mean) absolute mel-dB error after the top_db clamp."""
    d = np.abs(np.asarray(test_db, np.float64) - oracle_db)
    if d.size == 0:
        return 0.0, 0.0
    return float(d.max()), float(d.mean())


def mfcc_rel_error(test: np.ndarray, oracle_c: np.ndarray) -> float:
    """Max |test - oracle| normalised by max |oracle| over the clip."""
    oracle_c = np.asarray(oracle_c, np.float64)
    if oracle_c.size == 0:
        return 0.0
    scale = max(float(np.abs(oracle_c).max()), 1e-30)
    return float(np.abs(np.asarray(test, np.float64) - oracle_c).max() / scale)
