"""GPU parity: the CUDA path through the C ABI against the FP64 oracle and the
reference's golden vectors.

Tolerances (stated per test):
  * golden vectors -- the reference's own (rtol=atol=1e-4; 5e-4 for the
    fmin=300/fmax=8000 MFCC), Tests/test_parity_*.py;
  * mel-dB vs FP64 oracle -- 1e-3 dB max abs after the top_db floor;
  * MFCC vs FP64 oracle -- 1e-4 of max |c| per clip;
  * linear spectra vs FP64 oracle -- 2e-5 of the frame-set maximum (float32 FFT);
  * frame counts, padding and shapes -- exact.
"""

import numpy as np
import pytest

import metalmom_b200 as M
from metalmom_b200 import synth
from goldens import golden, signal_440
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SR = 22050
DB_TOL = 1e-3
MFCC_TOL = 1e-4


def _db_from_power(P, top_db=80.0):
    return O.power_to_db(np.asarray(P, np.float64), 1.0, 1e-10, top_db)


# ---------------------------------------------------------------------------
# golden vectors (the reference's tests, run against the CUDA path)
# ---------------------------------------------------------------------------

def test_stft_golden():
    y = signal_440()
    exp = golden("stft_440hz_default_magnitude")
    got = M.stft(y, n_fft=2048, hop_length=512, win_length=2048, center=True)
    assert got.shape == exp.shape and got.dtype == np.float32
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4)
    mid = got.shape[1] // 2
    assert np.argmax(got[:, mid]) == np.argmax(exp[:, mid])
    assert 0.99 < np.sum(got.astype(np.float64) ** 2) / np.sum(exp.astype(np.float64) ** 2) < 1.01


@pytest.mark.parametrize("name,kw", [
    ("mel_spectrogram_440hz_default", dict()),
    ("mel_spectrogram_440hz_40_1024", dict(n_fft=1024, n_mels=40)),
    ("mel_spectrogram_440hz_64_fmin300_fmax8000", dict(n_fft=2048, n_mels=64, fmin=300, fmax=8000)),
])
def test_melspectrogram_golden(name, kw):
    exp = golden(name)
    got = M.melspectrogram(y=signal_440(), sr=SR, **kw)
    assert got.shape == exp.shape and got.dtype == np.float32
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4)
    assert np.all(got >= 0)


@pytest.mark.parametrize("name,kw,tol", [
    ("mfcc_440hz_default", dict(), 1e-4),
    ("mfcc_440hz_13_1024", dict(n_mfcc=13, n_fft=1024, n_mels=40), 1e-4),
    ("mfcc_440hz_20_64_fmin300_fmax8000", dict(n_mfcc=20, n_fft=2048, n_mels=64, fmin=300, fmax=8000), 5e-4),
])
def test_mfcc_golden(name, kw, tol):
    exp = golden(name)
    got = M.mfcc(y=signal_440(), sr=SR, **kw)
    assert got.shape == exp.shape and got.dtype == np.float32
    np.testing.assert_allclose(got, exp, rtol=tol, atol=tol)
    assert np.all(np.isfinite(got))


def test_db_goldens():
    S = golden("stft_440hz_default_magnitude").astype(np.float32)
    np.testing.assert_allclose(M.amplitude_to_db(S, ref=np.max), golden("stft_440hz_amplitude_db"),
                               rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(M.amplitude_to_db(S, ref=1.0), golden("stft_440hz_amplitude_db_ref1"),
                               rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(M.power_to_db(S ** 2, ref=np.max), golden("stft_440hz_power_db"),
                               rtol=1e-4, atol=1e-4)


# ---------------------------------------------------------------------------
# FP64 oracle, across every supported FFT size and the padding/window cases
# ---------------------------------------------------------------------------

ALL_NFFT = [2 ** k for k in range(0, 16)]


@pytest.mark.parametrize("n_fft", ALL_NFFT)
def test_stft_all_sizes_vs_oracle(n_fft):
    rng = np.random.default_rng(n_fft)
    L = max(3 * n_fft + 17, 64)
    y = rng.standard_normal(L).astype(np.float32)
    hop = max(1, n_fft // 4)
    got = M.stft(y, n_fft=n_fft, hop_length=hop)
    exp = O.stft_magnitude(y, n_fft, hop, n_fft, True)
    assert got.shape == exp.shape == (n_fft // 2 + 1, O.n_frames(L, n_fft, hop, True))
    err = np.abs(got - exp).max() / exp.max()
    assert err < 2e-5, err


@pytest.mark.parametrize("n_fft,hop,win,center,L", [
    (2048, 512, 2048, True, 661500 // 10),
    (2048, 512, 2048, False, 50000),
    (512, 160, 400, True, 16000),      # window shorter than n_fft (centred, zero-padded)
    (2048, 512, 4096, True, 22050),    # window longer than n_fft (centre-truncated)
    (1024, 4096, 1024, True, 22050),   # hop longer than n_fft
    (2048, 441, 2048, True, 30001),    # odd hop: unaligned frame starts
    (1024, 256, 1024, True, 1),        # single sample, centred -> 1 frame
    (1024, 256, 1024, True, 300),      # shorter than n_fft/2
    (4096, 1024, 4096, True, 123457),
    (256, 64, 200, False, 9999),
])
def test_stft_cases_vs_oracle(n_fft, hop, win, center, L):
    y = synth.music_clip(L, SR, seed=L + n_fft)
    got = M.stft(y, n_fft=n_fft, hop_length=hop, win_length=win, center=center)
    exp = O.stft_magnitude(y, n_fft, hop, win, center)
    assert got.shape == exp.shape
    if exp.size:
        assert np.abs(got - exp).max() <= 2e-5 * max(exp.max(), 1e-30)


@pytest.mark.parametrize("power", [2.0, 1.0, 1.5])
def test_mel_power_variants_vs_oracle(power):
    y = synth.music_clip(44100, SR, seed=7)
    got = M.melspectrogram(y, sr=SR, n_fft=2048, hop_length=512, power=power)
    exp = O.melspectrogram(y, SR, 2048, 512, 2048, True, power, 128)
    assert got.shape == exp.shape
    assert np.abs(got - exp).max() <= 1e-5 * exp.max()
    if power == 2.0:
        mx, _ = O.mel_db_error(_db_from_power(got), _db_from_power(exp))
        assert mx < DB_TOL, mx


@pytest.mark.parametrize("sr,n_fft,hop,win,n_mels,n_mfcc,fmin,fmax,L", [
    (22050, 2048, 512, 2048, 128, 20, 0.0, None, 661500),   # the 30 s workload clip
    (16000, 512, 160, 400, 80, 13, 20.0, 8000.0, 160000),   # speech front end
    (44100, 4096, 1024, 4096, 64, 20, 0.0, None, 441000),
    (22050, 1024, 256, 1024, 40, 40, 0.0, None, 22050),     # n_mfcc == n_mels
    (22050, 2048, 512, 2048, 40, 200, 0.0, None, 22050),    # n_mfcc > n_mels -> capped
    (22050, 256, 64, 256, 32, 1, 0.0, None, 5000),          # single coefficient
])
def test_mfcc_and_meldb_vs_oracle(sr, n_fft, hop, win, n_mels, n_mfcc, fmin, fmax, L):
    y = (synth.speech_clip if sr == 16000 else synth.music_clip)(L, sr, seed=L ^ n_fft)
    got = M.mfcc(y, sr=sr, n_mfcc=n_mfcc, n_fft=n_fft, hop_length=hop, win_length=win,
                 n_mels=n_mels, fmin=fmin, fmax=fmax)
    exp = O.mfcc(y, sr, n_mfcc, n_fft, hop, win, n_mels, fmin, fmax, True)
    assert got.shape == exp.shape == (min(n_mfcc, n_mels), O.n_frames(L, n_fft, hop, True))
    assert O.mfcc_rel_error(got, exp) < MFCC_TOL
    mel = M.melspectrogram(y, sr=sr, n_fft=n_fft, hop_length=hop, win_length=win, n_mels=n_mels,
                           fmin=fmin, fmax=fmax)
    mx, _ = O.mel_db_error(_db_from_power(mel),
                           O.mel_db(y, sr, n_fft, hop, win, True, n_mels, fmin, fmax))
    assert mx < DB_TOL, mx


def test_power_to_db_vs_oracle():
    rng = np.random.default_rng(3)
    S = (rng.random((300, 77)) ** 6).astype(np.float32)
    for top_db in (80.0, 30.0, None):
        got = M.power_to_db(S, ref=1.0, top_db=top_db)
        exp = O.power_to_db(S.astype(np.float64), 1.0, 1e-10, top_db)
        assert np.abs(got - exp).max() < 1e-4
    got = M.amplitude_to_db(S, ref=np.max, top_db=60.0)
    assert got.min() >= got.max() - 60.0 - 1e-4


# ---------------------------------------------------------------------------
# edge cases the reference tests (EdgeCaseTests.swift, test_bridge_errors.py)
# ---------------------------------------------------------------------------

def test_silence_and_constant():
    z = np.zeros(22050, np.float32)
    assert np.all(M.stft(z) == 0.0)
    assert np.max(M.melspectrogram(z)) < 1e-10
    c = M.mfcc(z)
    assert np.all(np.isfinite(c))
    # c0 is -100 dB * sqrt(128) = -1131: the MFCC bar is relative to max |c|
    assert O.mfcc_rel_error(c, O.mfcc(z, SR, 20, 2048, 512, 2048, 128)) < MFCC_TOL
    one = np.ones(22050, np.float32)
    S = M.stft(one)
    mid = S.shape[1] // 2
    assert S[0, mid] > S[1:, mid].mean()


def test_nan_and_inf_inputs_do_not_crash():
    y = np.zeros(4096, np.float32)
    y[100] = np.nan
    y[500] = np.nan
    S = M.stft(y)
    assert S.shape == (1025, 9)
    y2 = np.zeros(4096, np.float32)
    y2[200] = np.inf
    y2[300] = -np.inf
    assert M.stft(y2).shape == (1025, 9)
    m = M.melspectrogram(y)
    assert m.shape == (128, 9)
    c = M.mfcc(y)
    assert c.shape == (20, 9)
    big = np.full(4096, np.finfo(np.float32).max / 1000, np.float32)
    assert M.stft(big).shape == (1025, 9)


def test_int_input_and_short_signal():
    assert M.stft(np.ones(2048, dtype=np.int32)).dtype == np.float32
    y = np.sin(np.arange(10, dtype=np.float32))
    S = M.stft(y)
    assert S.shape == (1025, 1)
    np.testing.assert_allclose(S, O.stft_magnitude(y, 2048, 512, 2048, True), atol=1e-5)


def test_buffer_freed_when_reshape_fails():
    from metalmom_b200._native import ffi, lib
    from metalmom_b200._bridge import take_buffer
    ctx = lib.mm_init()
    try:
        y = np.sin(np.arange(4096, dtype=np.float32))
        p = ffi.new("MMSTFTParams*")
        p.n_fft, p.hop_length, p.win_length, p.center = 2048, 512, 2048, 1
        out = ffi.new("MMBuffer*")
        assert lib.mm_stft(ctx, ffi.cast("const float*", y.ctypes.data), len(y), 22050, p, out) == 0
        assert out.count > 0
        out.shape[0] = 9999
        out.shape[1] = 9999
        with pytest.raises(ValueError):
            take_buffer(out)
        assert out.data == ffi.NULL
    finally:
        lib.mm_destroy(ctx)


# ---------------------------------------------------------------------------
# batching: uneven clips in one launch == per-clip calls; plans + graphs
# ---------------------------------------------------------------------------

def test_mfcc_batch_matches_single_clip_calls():
    rng = np.random.default_rng(11)
    lens = [int(x) for x in rng.integers(1, 90000, 9)] + [1, 1023, 1024, 1025]
    clips = [synth.music_clip(L, SR, seed=i) for i, L in enumerate(lens)]
    outs = M.mfcc_batch(clips, sr=SR, n_fft=2048, hop_length=512)
    for c, o in zip(clips, outs):
        single = M.mfcc(c, sr=SR, n_fft=2048, hop_length=512)
        assert o.shape == single.shape
        np.testing.assert_array_equal(o, single)
        exp = O.mfcc(c, SR, 20, 2048, 512, 2048, 128)
        assert O.mfcc_rel_error(o, exp) < MFCC_TOL


def test_reflect_padding_vs_oracle():
    clips = [synth.music_clip(L, SR, seed=L) for L in (5000, 22050, 1500)]
    outs = M.mfcc_batch(clips, sr=SR, n_fft=2048, hop_length=512, pad_mode="reflect")
    for c, o in zip(clips, outs):
        exp = O.mfcc(c, SR, 20, 2048, 512, 2048, 128, pad_mode=O.PAD_REFLECT)
        assert O.mfcc_rel_error(o, exp) < MFCC_TOL
    const = M.mfcc_batch(clips[:1], sr=SR, n_fft=2048, hop_length=512)[0]
    assert np.abs(const - outs[0]).max() > 1e-2  # the two paddings really differ


def test_plan_graph_replay_and_host_io():
    rng = np.random.default_rng(5)
    lens = [int(x) for x in rng.integers(20000, 120000, 6)]
    clips = [synth.music_clip(L, SR, seed=100 + i) for i, L in enumerate(lens)]
    ref = M.mfcc_batch(clips, sr=SR)
    with M.Plan(lens, sr=SR) as plan:
        assert plan.frames == [r.shape[1] for r in ref]
        assert plan.kernel_launches == 3
        a = plan.execute_host(clips)
        b = plan.execute_host(clips)
        for x, y_, r in zip(a, b, ref):
            np.testing.assert_array_equal(x, y_)
            np.testing.assert_array_equal(x, r)


def _uneven_group(rng):
    """A parameter group of the uneven-batch workload: sr 22050/44100, n_fft
    1024/2048/4096 with hop n_fft/4, 64/128 mels, 20 MFCC."""
    n_fft = int(rng.choice([1024, 2048, 4096]))
    return dict(sr=int(rng.choice([22050, 44100])), n_fft=n_fft, hop_length=n_fft // 4,
                n_mels=int(rng.choice([64, 128])), n_mfcc=20)


@pytest.mark.parametrize("max_per_branch", [0, 4])
def test_grouped_plan_uneven_mixed_groups(max_per_branch):
    """Clips with their own parameter groups in one graph: equal to per-clip
    calls (bitwise) through host I/O and through graph replay."""
    rng = np.random.default_rng(40 + max_per_branch)
    params, clips = [], []
    for i in range(30):
        g = _uneven_group(rng) if i % 5 else dict(sr=16000, n_fft=512, hop_length=160, win_length=400,
                                                    n_mels=80, n_mfcc=13, fmin=20.0, fmax=8000.0)
        L = int(rng.integers(1, 4 * g["sr"]))
        params.append(g)
        clips.append((synth.speech_clip if g["sr"] == 16000 else synth.music_clip)(L, g["sr"], seed=500 + i))
    with M.Plan([len(c) for c in clips], clip_params=params, max_clips_per_branch=max_per_branch) as plan:
        n_groups = len({tuple(sorted(g.items())) for g in params})
        assert plan.branches >= n_groups
        if max_per_branch:
            assert plan.branches > n_groups
        outs = plan.execute_host(clips)
        again = plan.execute_host(clips)
        plan.execute()
    for c, g, o, o2 in zip(clips, params, outs, again):
        ref = M.mfcc_batch([c], **g)[0]
        assert o.shape == ref.shape
        np.testing.assert_array_equal(o, ref)
        np.testing.assert_array_equal(o2, ref)
    for c, g, o in list(zip(clips, params, outs))[:6]:
        exp = O.mfcc(c, g["sr"], g["n_mfcc"], g["n_fft"], g["hop_length"], g.get("win_length", g["n_fft"]),
                     g["n_mels"], g.get("fmin", 0.0), g.get("fmax"))
        if exp.size:
            assert O.mfcc_rel_error(o, exp) < MFCC_TOL


def test_grouped_plan_graph_replay_on_device_inputs():
    import torch
    rng = np.random.default_rng(77)
    params = [_uneven_group(rng) for _ in range(12)]
    clips = [synth.music_clip(int(rng.integers(3000, 3 * g["sr"])), g["sr"], seed=900 + i)
             for i, g in enumerate(params)]
    with M.Plan([len(c) for c in clips], clip_params=params, max_clips_per_branch=3) as plan:
        base = plan.device_input
        for c, off in zip(clips, plan.in_offsets):
            dst = torch.as_tensor(_DevFloats(base + 4 * off, len(c)), device="cuda")
            dst.copy_(torch.from_numpy(c).cuda())
        torch.cuda.synchronize()
        plan.execute()
        torch.cuda.synchronize()
        for c, g, off, r, f in zip(clips, params, plan.out_offsets, plan.clip_rows, plan.frames):
            got = torch.as_tensor(_DevFloats(plan.device_output + 4 * off, r * f), device="cuda").cpu().numpy()
            np.testing.assert_array_equal(got.reshape(r, f), M.mfcc_batch([c], **g)[0])


class _DevFloats:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 2}


# ---------------------------------------------------------------------------
# launch variants (autotuner search space): every variant is parity-checked
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("n_fft", [256, 512, 1024, 2048, 4096, 8192])
def test_every_launch_variant_vs_oracle(n_fft):
    y = synth.music_clip(3 * 22050 + 123, SR, seed=n_fft)
    exp = O.mfcc(y, SR, 20, n_fft, n_fft // 4, n_fft, 64)
    exp_mel = O.melspectrogram(y, SR, n_fft, n_fft // 4, n_fft, True, 2.0, 64)
    old = M.tune_get(n_fft)
    try:
        for v in range(4):
            M.tune_set(n_fft, v)
            got = M.mfcc(y, sr=SR, n_fft=n_fft, hop_length=n_fft // 4, n_mels=64)
            assert O.mfcc_rel_error(got, exp) < MFCC_TOL, (v, O.mfcc_rel_error(got, exp))
            mel = M.melspectrogram(y, sr=SR, n_fft=n_fft, hop_length=n_fft // 4, n_mels=64)
            assert np.abs(mel - exp_mel).max() <= 1e-5 * exp_mel.max(), v
    finally:
        M.tune_set(n_fft, old)


@pytest.mark.parametrize("n_fft,win,hop,pad_mode", [
    (2048, 2048, 512, "constant"),
    (2048, 2048, 441, "reflect"),   # odd hop: frame starts alternate between even and odd samples
    (1024, 1024, 256, "constant"),
    (512, 400, 160, "constant"),    # window shorter than n_fft
    (512, 512, 128, "reflect"),
    (256, 256, 64, "constant"),
    (4096, 4096, 1024, "constant"),  # one frame per warp pair
    (4096, 4096, 1001, "reflect"),
    (4096, 3000, 700, "constant"),
])
def test_warp_kernel_uneven_batch_vs_oracle(n_fft, win, hop, pad_mode):
    """Variant 3 (one warp per frame, a warp pair for n_fft 4096) on uneven
    clips: clips shorter than a frame, clips whose start is not 8-byte aligned
    in the batch buffer, and frames that reach into the padding on both ends."""
    rng = np.random.default_rng(n_fft + hop)
    lens = [1, 3, n_fft // 2 + 1, n_fft - 1, n_fft + 1, 5 * n_fft + 3] + \
           [int(x) for x in rng.integers(1000, 60000, 5)]
    if pad_mode == "reflect":
        lens = [L for L in lens if L > n_fft // 2]  # reflect needs L > n_fft/2
    clips = [synth.music_clip(L, SR, seed=1000 + i) for i, L in enumerate(lens)]
    old = M.tune_get(n_fft)
    try:
        M.tune_set(n_fft, 3)
        outs = M.mfcc_batch(clips, sr=SR, n_fft=n_fft, hop_length=hop, win_length=win, n_mels=64,
                            pad_mode=pad_mode)
        single = M.mfcc(clips[-1], sr=SR, n_fft=n_fft, hop_length=hop, win_length=win, n_mels=64) \
            if pad_mode == "constant" else None
    finally:
        M.tune_set(n_fft, old)
    pm = O.PAD_REFLECT if pad_mode == "reflect" else O.PAD_CONSTANT
    for c, o in zip(clips, outs):
        exp = O.mfcc(c, SR, 20, n_fft, hop, win, 64, pad_mode=pm)
        assert o.shape == exp.shape
        if exp.size:
            assert O.mfcc_rel_error(o, exp) < MFCC_TOL, (len(c), O.mfcc_rel_error(o, exp))
    if single is not None:
        np.testing.assert_array_equal(single, outs[-1])


def test_autotune_picks_a_variant_and_keeps_parity():
    res = M.autotune(clip_samples=22050 * 5, n_clips=8, reps=3, sr=SR, n_fft=2048, hop_length=512)
    # n_fft 2048 on the MFCC path: variants 0-3 and the tensor-core kernel (5)
    assert res["best"] in (0, 1, 2, 3, 5) and sorted(res["ms"]) == [0, 1, 2, 3, 5]
    assert all(m > 0 for m in res["ms"].values())
    assert M.tune_get(2048) == res["best"]
    y = synth.music_clip(22050 * 4, SR, seed=9)
    got = M.mfcc(y, sr=SR)
    assert O.mfcc_rel_error(got, O.mfcc(y, SR, 20, 2048, 512, 2048, 128)) < MFCC_TOL


@pytest.mark.parametrize("length", [22048, 22051])
def test_plan_host_io_from_one_batch_array(length):
    """Clips passed as rows of one host array (their buffers adjacent) are
    uploaded and downloaded as merged runs; the results equal those from
    separate buffers bitwise.  Length 22051 leaves a 4-float alignment gap
    between the device slots, so no run forms there."""
    n = 12
    batch = np.stack([synth.music_clip(length, SR, seed=900 + i) for i in range(n)])
    sep = [row.copy() for row in batch]
    with M.Plan([length] * n, clip_params=[dict(sr=SR, n_fft=2048, hop_length=512)] * n,
                max_clips_per_branch=5) as plan:
        assert plan.branches == 3
        ref = plan.execute_host(sep)
        out = np.empty((n,) + ref[0].shape, np.float32)
        got = plan.execute_host(list(batch), list(out))
    for i in range(n):
        np.testing.assert_array_equal(got[i], ref[i])
        np.testing.assert_array_equal(out[i], ref[i])


@pytest.mark.parametrize("n_fft,hop,n_mels", [(2048, 512, 128), (512, 128, 120), (2048, 512, 600)])
def test_nonfinite_samples_floor_their_frames(n_fft, hop, n_mels):
    """A NaN or an infinite sample makes every band of the frames that hold it
    non-finite, which vDSP_vthr maps to amin (-100 dB) before the top_db floor;
    the other frames are untouched.  (2048, 128): the lane walk's check;
    (512, 120) and (2048, 600): too many filterbank parts for the lane tables,
    so the packed rows and their own check.)"""
    y = synth.music_clip(22050, SR, seed=31)
    y[5000] = np.nan
    y[15000] = np.inf
    y[18000] = -np.inf
    with np.errstate(all="ignore"):
        exp = O.mfcc(y, SR, 20, n_fft, hop, n_fft, n_mels)
    got = M.mfcc(y, sr=SR, n_fft=n_fft, hop_length=hop, n_mels=n_mels)
    assert got.shape == exp.shape and np.isfinite(got).all()
    assert O.mfcc_rel_error(got, exp) < MFCC_TOL


@pytest.mark.parametrize("n_fft,n_mels,fmin,fmax", [
    (2048, 1, 0.0, None),        # one band: its segment runs through every lane
    (2048, 20, 0.0, None),       # wide bands: segments over several lanes
    (2048, 64, 300.0, 4000.0),   # bins past fmax carry the last segment to the end
    (2048, 256, 0.0, None),
    (2048, 400, 0.0, None),      # 32 walking lanes: under their 480 part slots
    (2048, 600, 0.0, None),      # over them: packed rows over the 36-float padded spectrum
    (1024, 64, 0.0, None),
    (512, 100, 0.0, None),       # lane tables near their slot limit
    (512, 120, 0.0, None),       # over it: packed rows
    (256, 40, 50.0, None),
    (4096, 1, 0.0, None),
    (4096, 128, 0.0, None),
    (4096, 64, 300.0, 4000.0),
    (4096, 700, 0.0, None),
    (4096, 1100, 0.0, None),     # more parts than the lane tables hold: packed rows
])
def test_warp_kernel_filterbank_shapes_vs_oracle(n_fft, n_mels, fmin, fmax):
    """The warp kernel's filterbank walk (parts per lane, segment heads that
    take the parts of the lanes they run into, two-slot bands) on filterbanks
    that stress its tables; n_mfcc = n_mels where the DCT allows it, so the
    MFCC bound also bounds the log-mel rows."""
    y = synth.music_clip(4 * SR + 77, SR, seed=n_fft + n_mels)
    n_mfcc = min(n_mels, 32)
    exp = O.mfcc(y, SR, n_mfcc, n_fft, n_fft // 4, n_fft, n_mels, fmin, fmax)
    # n_fft 4096: the CTA-tile kernel (variant 2) walks the same tables
    for v in ((2, 3) if n_fft == 4096 else (3,)):
        old = M.tune_get(n_fft)
        try:
            M.tune_set(n_fft, v)
            got = M.mfcc(y, sr=SR, n_mfcc=n_mfcc, n_fft=n_fft, hop_length=n_fft // 4, n_mels=n_mels,
                         fmin=fmin, fmax=fmax)
        finally:
            M.tune_set(n_fft, old)
        assert got.shape == exp.shape
        assert O.mfcc_rel_error(got, exp) < MFCC_TOL, (v, O.mfcc_rel_error(got, exp))


@pytest.mark.parametrize("n_mels", [128, 1100])
def test_warp_pair_kernel_nonfinite_samples(n_mels):
    """n_fft 4096 on the warp-pair kernel: non-finite samples floor their
    frames through the lane walk's check (128 bands) and the packed rows'
    check (1100 bands)."""
    y = synth.music_clip(3 * SR, SR, seed=37)
    y[9000] = np.nan
    y[40000] = np.inf
    old = M.tune_get(4096)
    try:
        M.tune_set(4096, 3)
        got = M.mfcc(y, sr=SR, n_mfcc=32, n_fft=4096, hop_length=1024, n_mels=n_mels)
    finally:
        M.tune_set(4096, old)
    with np.errstate(all="ignore"):
        exp = O.mfcc(y, SR, 32, 4096, 1024, 4096, n_mels)
    assert got.shape == exp.shape and np.isfinite(got).all()
    assert O.mfcc_rel_error(got, exp) < MFCC_TOL


def test_large_finite_samples_are_not_flagged_non_finite():
    """Broadband samples of ~1e17: every bin power is finite (~3e37) although
    a thread's bins sum past the float32 range.  The frames' non-finite checks
    accumulate |X|^2 * 0, so no frame is floored as non-finite: mel power and
    MFCC follow the oracle on the CTA-tile kernel (variant 0) and the warp
    kernel (variant 3)."""
    rng = np.random.default_rng(11)
    y = (rng.standard_normal(2 * SR) * 1e17).astype(np.float32)
    exp = O.mfcc(y, SR, 20, 2048, 512, 2048, 128)
    exp_mel = O.melspectrogram(y, SR, 2048, 512, 2048, True, 2.0, 128)
    assert np.isfinite(exp_mel).all() and exp_mel.max() > 1e35
    old = M.tune_get(2048)
    try:
        for v in (0, 3):
            M.tune_set(2048, v)
            got = M.mfcc(y, sr=SR)
            assert O.mfcc_rel_error(got, exp) < MFCC_TOL, (v, O.mfcc_rel_error(got, exp))
    finally:
        M.tune_set(2048, old)
    mel = M.melspectrogram(y, sr=SR)
    assert np.isfinite(mel).all()
    assert np.abs(mel - exp_mel).max() <= 1e-5 * exp_mel.max()


def test_batch_mixing_short_and_long_clips_matches_single_calls():
    """Clips of 1 MB and more are uploaded from the caller's buffer, shorter
    ones through pinned staging whose upload spans the whole signal region;
    in a batch that mixes both, every clip's result equals its single-clip
    result bitwise."""
    lens = [1000, 300000, 5000, 400000, 262144, 262143]
    clips = [synth.music_clip(L, SR, seed=70 + i) for i, L in enumerate(lens)]
    outs = M.mfcc_batch(clips, sr=SR, n_fft=2048, hop_length=512)
    for c, o in zip(clips, outs):
        np.testing.assert_array_equal(o, M.mfcc(c, sr=SR, n_fft=2048, hop_length=512))
    exp = O.mfcc(clips[1], SR, 20, 2048, 512, 2048, 128)
    assert O.mfcc_rel_error(outs[1], exp) < MFCC_TOL


@pytest.mark.parametrize("n_mels", [64, 80, 128])
@pytest.mark.parametrize("n_mfcc", [1, 2, 5, 9, 13, 20, 24, 28, 32])
def test_folded_dct_every_coefficient_group_vs_oracle(n_mels, n_mfcc):
    """The folded cp.async DCT (64, 80 and 128 bands) for every number of
    accumulators per coefficient group (KQ = ceil(ceil(n_mfcc / 2) / 2), 1..8)
    and a clip whose last 64-frame tile is partial; n_mfcc above 32 falls to
    the chunked kernels and is covered above."""
    y = synth.music_clip(3 * SR + 1234, SR, seed=n_mels * 100 + n_mfcc)
    got = M.mfcc(y, sr=SR, n_mfcc=n_mfcc, n_fft=2048, hop_length=512, n_mels=n_mels)
    exp = O.mfcc(y, SR, n_mfcc, 2048, 512, 2048, n_mels)
    assert got.shape == exp.shape
    assert O.mfcc_rel_error(got, exp) < MFCC_TOL, O.mfcc_rel_error(got, exp)
