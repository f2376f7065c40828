"""mm_mfcc_noalloc: the MFCC entry point that allocates no device memory.

It serves callers that cannot allocate while they run -- code inside another
framework's memory pool or under a hard memory budget, real-time audio threads
that may not block in the allocator, plugin hosts that forbid cudaMalloc --
by taking all scratch from a fixed array built into the library.  Checked here
through the C ABI against mm_mfcc (the existing entry point) on two calls in a
row, with the MFCC tolerance the other tests use (1e-4 of max |c|).  The file
name makes pytest collect it last.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MFCC_TOL = 1e-4


def _noalloc(y_dev, n, out_dev, stream, **kw):
    from metalmom_b200._native import ffi, lib
    p = dict(sr=22050, n_mfcc=20, n_fft=2048, hop=512, win=2048, n_mels=128, fmin=0.0, fmax=0.0, center=1)
    p.update(kw)
    return lib.mm_mfcc_noalloc(ffi.cast("const float*", y_dev), n, p["sr"], p["n_mfcc"], p["n_fft"],
                               p["hop"], p["win"], p["n_mels"], p["fmin"], p["fmax"], p["center"],
                               ffi.cast("float*", out_dev), ffi.cast("void*", stream))


def test_noalloc_matches_mm_mfcc_on_two_calls():
    import torch
    import metalmom_b200 as M
    from metalmom_b200 import synth
    stream = torch.cuda.current_stream().cuda_stream
    # call 1: an aligned clip; call 2: a different clip read from a 4-byte offset
    a = synth.music_clip(3 * 22050 + 17, 22050, seed=1)
    b = synth.music_clip(5 * 22050, 22050, seed=2)
    for y, offset in ((a, 0), (b, 1)):
        ref = M.mfcc(y, sr=22050)
        rows, T = ref.shape
        host = np.concatenate([np.zeros(offset, np.float32), y])
        d_y = torch.from_numpy(host).cuda()
        d_out = torch.full((rows * T,), float("nan"), device="cuda")
        st = _noalloc(d_y.data_ptr() + 4 * offset, len(y), d_out.data_ptr(), stream)
        assert st == 0
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().reshape(rows, T)
        assert np.all(np.isfinite(got))
        err = np.abs(got.astype(np.float64) - ref).max() / np.abs(ref).max()
        assert err < MFCC_TOL, err


def test_noalloc_rejects_clips_beyond_its_scratch():
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    d_y = torch.zeros(4096, device="cuda")
    d_out = torch.zeros(16, device="cuda")
    # 40 001 frames x 128 mels x 4 bytes (20.5 MB) of log-mel scratch exceed the
    # 16 MiB array on their own: the call refuses before launching anything
    assert _noalloc(d_y.data_ptr(), 40000 * 512, d_out.data_ptr(), stream) == -1
    assert _noalloc(0, 4096, d_out.data_ptr(), stream) == -1
