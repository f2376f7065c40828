"""B200-native spectral front end with MetalMom's API.

``stft``, ``melspectrogram``, ``mfcc``, ``power_to_db`` and ``amplitude_to_db``
keep the names, defaults and error behaviour of MetalMom's Python package and
run on the GPU through ``libmetalmom.so``; ``mfcc_batch`` and ``Plan`` add a
batched, device-resident path and ``Server`` a continuously batching request
loop.
"""

from .core import istft, stft, stft_complex
from .feature import (amplitude_to_db, amplitude_to_db_device, delta, melspectrogram, mfcc, power_to_db,
                      power_to_db_device, stack_memory)
from .onset import onset_strength
from .batch import Plan, autotune, frontend_params, mfcc_batch, tune_get, tune_set
from .serve import Server

__all__ = ["stft", "stft_complex", "istft", "melspectrogram", "mfcc", "power_to_db", "amplitude_to_db",
           "power_to_db_device", "amplitude_to_db_device", "onset_strength", "delta", "stack_memory",
           "mfcc_batch", "Plan", "frontend_params", "autotune", "tune_get", "tune_set", "Server"]
