"""mm_mfcc_noalloc: the MFCC entry point that allocates no device memory.

It serves callers that cannot allocate while they run -- code inside another
framework's memory pool or under a hard memory budget, real-time audio threads
that may not block in the allocator, plugin hosts that forbid cudaMalloc -- by
taking all scratch from a fixed array built into the library.

Checked here through the C ABI, on two calls in a row per parameter set (the
second repeats the parameters, so it runs on the tables the first left in the
array), against the FP64 oracle and against mm_mfcc (the existing entry point)
with the MFCC tolerance the other tests use (1e-4 of max |c|), over the kernel
families the library picks by size: the warp kernel (n_fft 2048), the
warp-pair kernel (4096), the CTA-tile kernels (256, 1024, 512 with a shorter
window) and the direct-DFT kernel (16), centred and not, from aligned and
4-byte-offset signals.  The device's free memory is the same before and after
a run of calls.  The file name makes pytest collect it last.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MFCC_TOL = 1e-4

# (sr, n_fft, hop, win, n_mels, n_mfcc, fmin, fmax, center, offset in floats)
CASES = [
    (22050, 2048, 512, 2048, 128, 20, 0.0, 0.0, 1, 0),
    (22050, 2048, 512, 2048, 128, 20, 0.0, 0.0, 1, 1),
    (44100, 4096, 1024, 4096, 128, 20, 0.0, 0.0, 1, 0),
    (22050, 1024, 256, 1024, 64, 20, 0.0, 0.0, 0, 1),
    (16000, 256, 64, 256, 40, 13, 0.0, 0.0, 1, 1),
    (16000, 512, 160, 400, 80, 13, 20.0, 8000.0, 1, 0),
    (8000, 16, 4, 16, 6, 5, 0.0, 0.0, 1, 0),
]
IDS = ["2048", "2048-off1", "4096", "1024-nocenter-off1", "256-40mels-off1", "512-win400", "16-tiny"]


def _noalloc(y_dev, n, out_dev, stream, c):
    from metalmom_b200._native import ffi, lib
    sr, n_fft, hop, win, n_mels, n_mfcc, fmin, fmax, center, _ = c
    return lib.mm_mfcc_noalloc(ffi.cast("const float*", y_dev), n, sr, n_mfcc, n_fft, hop, win, n_mels, fmin,
                               fmax, center, ffi.cast("float*", out_dev), ffi.cast("void*", stream))


def _run(y, c, stream):
    """One call through the C ABI; the signal sits `offset` floats into its
    device buffer.  Returns the [rows, frames] result."""
    import torch
    from oracle import oracle as O
    sr, n_fft, hop, win, n_mels, n_mfcc, fmin, fmax, center, offset = c
    T = O.n_frames(len(y), n_fft, hop, bool(center))
    rows = min(n_mfcc, n_mels)
    d_y = torch.from_numpy(np.concatenate([np.zeros(offset, np.float32), y])).cuda()
    d_out = torch.full((rows * T,), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(d_y.data_ptr() + 4 * offset, len(y), d_out.data_ptr(), stream, c) == 0
    torch.cuda.synchronize()
    return d_out.cpu().numpy().reshape(rows, T)


@pytest.mark.parametrize("c", CASES, ids=IDS)
def test_noalloc_matches_oracle_and_mm_mfcc_on_two_calls(c):
    import torch
    import metalmom_b200 as M
    from metalmom_b200 import synth
    from oracle import oracle as O
    sr, n_fft, hop, win, n_mels, n_mfcc, fmin, fmax, center, offset = c
    stream = torch.cuda.current_stream().cuda_stream
    kw = dict(sr=sr, n_mfcc=n_mfcc, n_fft=n_fft, hop_length=hop, win_length=win, n_mels=n_mels, fmin=fmin,
              fmax=fmax if fmax > 0 else None, center=bool(center))
    # two different clips, one call each, the same parameters
    for k, secs in enumerate((3.0, 5.0)):
        y = synth.music_clip(int(secs * sr) + 17 * k, sr, seed=10 * n_fft + k)
        got = _run(y, c, stream)
        exp = O.mfcc(y, sr, n_mfcc, n_fft, hop, win, n_mels, fmin, fmax if fmax > 0 else None, bool(center))
        assert got.shape == exp.shape
        assert np.all(np.isfinite(got))
        assert O.mfcc_rel_error(got, exp) < MFCC_TOL, (k, O.mfcc_rel_error(got, exp))
        ref = M.mfcc(y, **kw)
        assert O.mfcc_rel_error(got, ref) < MFCC_TOL, (k, O.mfcc_rel_error(got, ref))


def test_noalloc_leaves_device_free_memory_unchanged():
    import torch
    from metalmom_b200 import synth
    stream = torch.cuda.current_stream().cuda_stream
    bufs = []
    for c in CASES:
        sr = c[0]
        y = synth.music_clip(4 * sr, sr, seed=c[1])
        T = 1 + (len(y) + 2 * (c[1] // 2) - c[1]) // c[2] if c[8] else 1 + (len(y) - c[1]) // c[2]
        d_y = torch.from_numpy(np.concatenate([np.zeros(c[9], np.float32), y])).cuda()
        d_out = torch.empty(min(c[5], c[4]) * T, device="cuda")
        bufs.append((c, d_y, len(y), d_out))
    # every kernel of these calls once, so that lazy loading of their code is
    # behind us; then a full round of calls (each a new parameter set, so each
    # rebuilds its tables in the array) must leave free memory as it was
    for c, d_y, n, d_out in bufs:
        assert _noalloc(d_y.data_ptr() + 4 * c[9], n, d_out.data_ptr(), stream, c) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        for c, d_y, n, d_out in bufs:
            assert _noalloc(d_y.data_ptr() + 4 * c[9], n, d_out.data_ptr(), stream, c) == 0
            assert _noalloc(d_y.data_ptr() + 4 * c[9], n, d_out.data_ptr(), stream, c) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_clips_beyond_its_scratch():
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    c = CASES[0]
    n = 40000 * 512  # 40 001 frames x 128 mels x 4 bytes (20.5 MB) of log-mel rows > the 16 MiB array
    # a device buffer of the full claimed length, so that the call reads in
    # bounds even if it did not refuse
    d_y = torch.zeros(n, device="cuda")
    d_out = torch.zeros(20 * 40001, device="cuda")
    assert _noalloc(d_y.data_ptr(), n, d_out.data_ptr(), stream, c) == -1
    assert _noalloc(0, 4096, d_out.data_ptr(), stream, c) == -1
    torch.cuda.synchronize()
