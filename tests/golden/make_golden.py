"""Collect the reference's golden vectors for the spectral front end.

MetalMom pins its STFT / mel / MFCC / dB path (and the onset strength and
delta / stack_memory features built on it) against librosa-generated
``.npy`` files (``Tests/golden/``, written by ``scripts/generate_golden.py``
in the MetalMom project; librosa >= 0.11).  This script copies the files that
belong to that path into one compressed archive,
``tests/golden/reference_goldens.npz``, so the tests can run where the
MetalMom checkout is absent.  The mel filterbank goldens are stored sparsely
(row, column, value of each nonzero) to keep the archive small; the loader in
``tests/goldens.py`` restores them densely.

Usage (needs a MetalMom checkout, given as the argument or in
MM_REFERENCE_DIR):
    python tests/golden/make_golden.py /path/to/MetalMom
"""

import os
import sys

import numpy as np

DENSE = [
    "signal_440hz_22050sr",
    "stft_440hz_default_magnitude",
    "stft_440hz_amplitude_db",
    "stft_440hz_amplitude_db_ref1",
    "stft_440hz_power_db",
    "mel_spectrogram_440hz_default",
    "mel_spectrogram_440hz_40_1024",
    "mel_spectrogram_440hz_64_fmin300_fmax8000",
    "mfcc_440hz_default",
    "mfcc_440hz_13_1024",
    "mfcc_440hz_20_64_fmin300_fmax8000",
    # widening of the path: onset strength, delta / stack_memory on MFCC
    "onset_strength_440hz_default",
    "mfcc",
    "delta",
    "delta_delta",
    "stack_memory",
]
SPARSE = [
    "mel_filterbank_128_2048",
    "mel_filterbank_40_1024",
    "mel_filterbank_64_2048_300_8000",
]


def main(root: str) -> None:
    src = os.path.join(root, "Tests", "golden")
    arrays = {}
    for name in DENSE:
        arrays[name] = np.load(os.path.join(src, name + ".npy"))
    for name in SPARSE:
        a = np.load(os.path.join(src, name + ".npy"))
        r, c = np.nonzero(a)
        arrays[name + "__shape"] = np.array(a.shape, dtype=np.int64)
        arrays[name + "__row"] = r.astype(np.int32)
        arrays[name + "__col"] = c.astype(np.int32)
        arrays[name + "__val"] = a[r, c]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "reference_goldens.npz")
    np.savez_compressed(out, **arrays)
    print(f"wrote {out} ({os.path.getsize(out)} bytes, {len(DENSE) + len(SPARSE)} goldens)")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MM_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_golden.py <MetalMom checkout> (or set MM_REFERENCE_DIR)")
    main(ref)
