"""Seeded synthetic audio for the benchmark workloads and the tests.

No public dataset is involved: every workload is generated from a seed.

``music_clip`` -- sum of K ~ U{1..8} sinusoids (frequency U[50, 8000] Hz,
amplitude U[0.05, 0.5], random phase) + Gaussian noise (sigma 0.01) + 20
exponentially decaying clicks at uniform times (amplitude 0.5 with random
sign, decay constant 200 samples), clipped to [-1, 1].

``speech_clip`` -- harmonic stack (f0 U[80, 300] Hz, 10 harmonics with
amplitude 1/k) amplitude-modulated at 4 Hz (gain 0.5 + 0.5 sin), + Gaussian
noise (sigma 0.005), clipped to [-1, 1].
"""

import numpy as np

CLICK_AMP = 0.5
CLICK_TAU = 200.0
N_CLICKS = 20


def music_clip(n_samples: int, sr: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(n_samples, dtype=np.float64) / sr
    y = np.zeros(n_samples, dtype=np.float64)
    for _ in range(int(rng.integers(1, 9))):
        f = rng.uniform(50.0, 8000.0)
        a = rng.uniform(0.05, 0.5)
        ph = rng.uniform(0.0, 2.0 * np.pi)
        y += a * np.sin(2.0 * np.pi * f * t + ph)
    y += rng.normal(0.0, 0.01, n_samples)
    klen = int(CLICK_TAU * 8)
    kern = CLICK_AMP * np.exp(-np.arange(klen) / CLICK_TAU)
    for pos in rng.integers(0, max(n_samples, 1), N_CLICKS):
        sgn = 1.0 if rng.random() < 0.5 else -1.0
        end = min(n_samples, pos + klen)
        y[pos:end] += sgn * kern[:end - pos]
    return np.clip(y, -1.0, 1.0).astype(np.float32)


def speech_clip(n_samples: int, sr: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(n_samples, dtype=np.float64) / sr
    f0 = rng.uniform(80.0, 300.0)
    y = np.zeros(n_samples, dtype=np.float64)
    for k in range(1, 11):
        y += (1.0 / k) * np.sin(2.0 * np.pi * k * f0 * t + rng.uniform(0.0, 2.0 * np.pi))
    y *= 0.5 + 0.5 * np.sin(2.0 * np.pi * 4.0 * t)
    y *= 0.2
    y += rng.normal(0.0, 0.005, n_samples)
    return np.clip(y, -1.0, 1.0).astype(np.float32)
