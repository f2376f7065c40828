"""Loader for the reference's golden vectors (see golden/make_golden.py)."""

import os

import numpy as np

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                     "reference_goldens.npz")
_cache = {}


def golden(name: str) -> np.ndarray:
    """Return golden ``name`` (the reference's ``Tests/golden/<name>.npy``)."""
    if name in _cache:
        return _cache[name]
    z = np.load(_PATH)
    if name in z.files:
        arr = z[name]
    else:
        shape = tuple(int(s) for s in z[name + "__shape"])
        arr = np.zeros(shape, dtype=z[name + "__val"].dtype)
        arr[z[name + "__row"], z[name + "__col"]] = z[name + "__val"]
    _cache[name] = arr
    return arr


def signal_440() -> np.ndarray:
    return golden("signal_440hz_22050sr")
