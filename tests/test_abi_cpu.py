"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and keeps the reference's validation and empty-result rules
(MetalMom Bridge.swift:44-140, 267-492, 3695-3711; Tests/test_bridge_errors.py).
"""

import ctypes
import subprocess

import numpy as np
import pytest

from metalmom_b200 import _native
from metalmom_b200._native import ffi, lib
import metalmom_b200 as M


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_exports_every_header_symbol():
    names = _native.exported_names()
    assert len(names) >= 23
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # only the C ABI is exported
    assert all(n.startswith("mm_") for n in exported), sorted(exported)
    so = ctypes.CDLL(_native.LIB_PATH)
    for n in names:
        assert getattr(so, n) is not None


def test_struct_layout_matches_reference():
    assert ffi.sizeof("MMBuffer") == 88
    assert ffi.offsetof("MMBuffer", "ndim") == 72
    assert ffi.offsetof("MMBuffer", "count") == 80
    assert ffi.sizeof("MMSTFTParams") == 16
    assert lib.MM_OK == 0 and lib.MM_ERR_INVALID_INPUT == -1
    assert lib.MM_ERR_METAL_UNAVAILABLE == -2 and lib.MM_ERR_ALLOC_FAILED == -3
    assert lib.MM_ERR_INTERNAL == -4


def test_context_double_destroy_and_null():
    ctx = lib.mm_init()
    assert ctx != ffi.NULL
    lib.mm_destroy(ctx)
    lib.mm_destroy(ctx)
    lib.mm_destroy(ffi.NULL)
    lib.mm_buffer_free(ffi.NULL)


def _params(n_fft=2048, hop=512, win=2048, center=1):
    p = ffi.new("MMSTFTParams*")
    p.n_fft, p.hop_length, p.win_length, p.center = n_fft, hop, win, center
    return p


def test_invalid_inputs_return_minus_one():
    ctx = lib.mm_init()
    y = np.ones(22050, np.float32)
    yp = ffi.cast("const float*", y.ctypes.data)
    out = ffi.new("MMBuffer*")
    try:
        assert lib.mm_stft(ctx, ffi.NULL, 22050, 22050, _params(), out) == -1
        assert lib.mm_stft(ffi.NULL, yp, 22050, 22050, _params(), out) == -1
        assert lib.mm_stft(ctx, yp, 0, 22050, _params(), out) == -1
        assert lib.mm_stft(ctx, yp, 22050, 22050, ffi.NULL, out) == -1
        assert lib.mm_stft(ctx, yp, 22050, 22050, _params(), ffi.NULL) == -1
        assert lib.mm_stft(ctx, yp, 22050, 22050, _params(n_fft=1000, win=1000), out) == -1
        assert out.data == ffi.NULL
        assert lib.mm_mfcc(ctx, ffi.NULL, 10, 22050, 20, 2048, 512, 2048, 128, 0.0, 0.0, 1, out) == -1
        assert lib.mm_mfcc(ctx, yp, -5, 22050, 20, 2048, 512, 2048, 128, 0.0, 0.0, 1, out) == -1
        assert lib.mm_mel_spectrogram(ctx, yp, 0, 22050, 2048, 512, 2048, 1, 2.0, 128, 0.0, 0.0, out) == -1
        assert lib.mm_power_to_db(ctx, ffi.NULL, 10, 1.0, 1e-10, 80.0, out) == -1
        assert lib.mm_power_to_db(ctx, yp, 0, 1.0, 1e-10, 80.0, out) == -1
        assert lib.mm_amplitude_to_db(ctx, yp, 10, 1.0, 1e-5, 80.0, ffi.NULL) == -1
    finally:
        lib.mm_destroy(ctx)


def test_empty_results_need_no_gpu():
    """Empty outputs follow the reference: MM_OK, data NULL, shape [rows, 0]."""
    y = np.ones(8000, np.float32)
    # non power-of-two n_fft in mel/MFCC -> zero frames (EdgeCaseTests.swift:115-140)
    assert M.melspectrogram(y, n_fft=1000, n_mels=40).shape == (40, 0)
    assert M.mfcc(y, n_fft=1000, n_mfcc=13, n_mels=40).shape == (13, 0)
    # uncentered signal shorter than n_fft -> zero frames
    short = np.ones(100, np.float32)
    assert M.stft(short, center=False).shape == (1025, 0)
    # n_mels = 0 -> (0, n_frames) (EdgeCaseTests.swift:173-183)
    T = 1 + 8000 // 512
    assert M.melspectrogram(y, n_mels=0).shape == (0, T)
    assert M.mfcc(y, n_mfcc=0).shape == (0, T)


def test_empty_array_raises():
    with pytest.raises(RuntimeError, match="failed with status"):
        M.stft(np.array([], dtype=np.float32))


@pytest.mark.skipif(_have_gpu(), reason="checks the no-GPU status")
def test_no_gpu_is_reported_not_hidden():
    """Without a CUDA device the compute calls fail with -2; there is no CPU fallback."""
    y = np.ones(4096, np.float32)
    for fn in (lambda: M.stft(y), lambda: M.mfcc(y), lambda: M.melspectrogram(y),
               lambda: M.power_to_db(y), lambda: M.mfcc_batch([y, y])):
        with pytest.raises(RuntimeError, match="status -2"):
            fn()
    with pytest.raises(RuntimeError, match="status -2"):
        M.Plan([4096, 5000])
    with pytest.raises(RuntimeError, match="status -2"):
        M.Server()
    with pytest.raises(RuntimeError, match="status -2"):
        M.Plan([4096, 5000], clip_params=[dict(sr=22050), dict(sr=16000, n_fft=512)])


def test_untuned_launch_variants():
    """Before any autotuning: the warp kernels (variant 3) for n_fft 2048 and
    4096, the CTA-tile kernel (variant 0) for every other size; mm_tune_set
    validates its arguments and the setting round-trips."""
    assert [M.tune_get(1 << b) for b in range(4, 16)] == [0] * 7 + [3, 3] + [0] * 3
    assert lib.mm_tune_set(1000, 0) == -1 and lib.mm_tune_set(2048, 4) == -1 and lib.mm_tune_set(2048, -1) == -1
    M.tune_set(1024, 2)
    try:
        assert M.tune_get(1024) == 2
    finally:
        M.tune_set(1024, 0)
