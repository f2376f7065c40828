"""B200-native spectral front end with MetalMom's API.

``stft``, ``melspectrogram``, ``mfcc``, ``power_to_db`` and ``amplitude_to_db``
keep the names, defaults and error behaviour of MetalMom's Python package and
run on the GPU through ``libmetalmom.so``; ``mfcc_batch`` and ``Plan`` add a
batched, device-resident path and ``Server`` a continuously batching request
loop.

The names below are bound on first use: ``import metalmom_b200.synth`` (the
seeded workload generators) or ``metalmom_b200.shard`` loads no native code,
and the first API call loads ``libmetalmom.so`` (an import error names the
build command when it is missing; there is no fallback).
"""

import importlib

_API = {
    "stft": "core", "stft_complex": "core", "istft": "core",
    "melspectrogram": "feature", "mfcc": "feature", "power_to_db": "feature", "amplitude_to_db": "feature",
    "power_to_db_device": "feature", "amplitude_to_db_device": "feature", "delta": "feature",
    "stack_memory": "feature",
    "onset_strength": "onset",
    "mfcc_batch": "batch", "Plan": "batch", "frontend_params": "batch", "autotune": "batch",
    "tune_get": "batch", "tune_set": "batch",
    "Server": "serve",
}

__all__ = list(_API)


def __getattr__(name):
    mod = _API.get(name)
    if mod is None:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    value = getattr(importlib.import_module(f".{mod}", __name__), name)
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_API))
