"""Serving engine (mm_server_*): continuous batching with device-memory
admission.

Checked here:
  * every request's result is the same alone and in the mix -- bitwise equal
    to a single-clip mm_mfcc_batch call with the same parameters, and within
    the MFCC tolerance (1e-4 of max |c|) of the FP64 oracle;
  * requests that arrive while batches run are admitted (several batches
    launch, mixed parameter groups run together);
  * the device budget caps the memory of the batches in flight, and a request
    that alone exceeds it fails cleanly;
  * latency statistics are reported.
"""

import threading
import time

import numpy as np
import pytest

import metalmom_b200 as M
from metalmom_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MFCC_TOL = 1e-4

# parameter groups of the served workload: music 22.05 kHz, music 44.1 kHz
# with n_fft 1024 / 64 mels, speech 16 kHz (n_fft 512, win 400, hop 160)
GROUPS = [
    dict(sr=22050, n_fft=2048, hop_length=512, n_mels=128, n_mfcc=20),
    dict(sr=44100, n_fft=1024, hop_length=256, n_mels=64, n_mfcc=20),
    dict(sr=16000, n_fft=512, hop_length=160, win_length=400, n_mels=80, n_mfcc=13, fmin=20.0, fmax=8000.0),
    dict(sr=22050, n_fft=4096, hop_length=1024, n_mels=128, n_mfcc=20),
]


def _requests(n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        g = GROUPS[i % len(GROUPS)]
        L = int(rng.integers(g["n_fft"] // 2 + 1, 6 * g["sr"]))
        gen = synth.speech_clip if g["sr"] == 16000 else synth.music_clip
        reqs.append((gen(L, g["sr"], seed=seed * 1000 + i), g))
    return reqs


def _oracle(y, g):
    return O.mfcc(y, g["sr"], g["n_mfcc"], g["n_fft"], g["hop_length"], g.get("win_length", g["n_fft"]),
                  g["n_mels"], g.get("fmin", 0.0), g.get("fmax"))


def test_results_same_alone_and_in_the_mix():
    reqs = _requests(24, seed=1)
    with M.Server(max_inflight=3, max_batch_clips=5) as srv:
        ids = []

        def producer():
            # staggered arrivals: later requests come while earlier batches run
            for k, (y, g) in enumerate(reqs):
                ids.append(srv.submit(y, **g))
                if k % 4 == 3:
                    time.sleep(0.002)

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        mixed = [srv.result(i, timeout_ms=60000) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches_launched"] >= len(GROUPS)
    assert st["latency_p99_ms"] >= st["latency_p50_ms"] > 0.0
    for (y, g), got in zip(reqs, mixed):
        alone = M.mfcc_batch([y], **g)[0]
        assert got.shape == alone.shape
        np.testing.assert_array_equal(got, alone)
    for (y, g), got in list(zip(reqs, mixed))[:8]:
        assert O.mfcc_rel_error(got, _oracle(y, g)) < MFCC_TOL


def test_each_request_alone_through_the_server_matches_the_mix():
    reqs = _requests(8, seed=2)
    with M.Server(max_inflight=4) as srv:
        ids = [srv.submit(y, **g) for y, g in reqs]
        mixed = [srv.result(i) for i in ids]
    for (y, g), m in zip(reqs, mixed):
        with M.Server(max_inflight=1) as one:
            alone = one.result(one.submit(y, **g))
        np.testing.assert_array_equal(m, alone)


def test_budget_caps_memory_in_flight():
    reqs = _requests(12, seed=3)
    budget = 64 << 20  # a few clips at a time
    with M.Server(budget_bytes=budget, max_inflight=4) as srv:
        ids = [srv.submit(y, **g) for y, g in reqs]
        outs = [srv.result(i) for i in ids]
        st = srv.stats()
    assert 0 < st["peak_bytes_in_use"] <= budget
    assert st["completed"] == len(reqs)
    for (y, g), o in zip(reqs, outs):
        np.testing.assert_array_equal(o, M.mfcc_batch([y], **g)[0])


def test_request_larger_than_budget_fails_cleanly():
    y = synth.music_clip(22050 * 60, 22050, seed=5)
    with M.Server(budget_bytes=1 << 20) as srv:
        rid = srv.submit(y, sr=22050)
        with pytest.raises(RuntimeError, match="status -3"):
            srv.result(rid)
        small = synth.music_clip(4096, 22050, seed=6)
        out = srv.result(srv.submit(small, sr=22050))
        assert out.shape == (20, 9)


def test_poll_and_invalid_requests():
    with M.Server() as srv:
        with pytest.raises(RuntimeError, match="status -1"):
            srv.submit(np.zeros(10, np.float32), sr=22050, center=False)  # no frame
        rid = srv.submit(synth.music_clip(22050, 22050, seed=7), sr=22050)
        deadline = time.time() + 60
        out = None
        while out is None and time.time() < deadline:
            out = srv.poll(rid)
            time.sleep(0.001)
        assert out is not None and out.shape == (20, 44)
        with pytest.raises(RuntimeError):
            srv.poll(rid)  # delivered requests are forgotten


def test_borrowed_submits_equal_copied_submits():
    """mm_server_submit_borrowed (and its many-request form) reads the
    caller's (here pinned) buffers in place: the results are bitwise those of
    copied submits."""
    import torch
    reqs = _requests(12, seed=7)
    total = sum(len(y) for y, _ in reqs)
    buf = torch.empty(total, dtype=torch.float32).pin_memory().numpy()
    views, off = [], 0
    for y, _ in reqs:
        views.append(buf[off:off + len(y)])
        views[-1][:] = y
        off += len(y)
    with M.Server(max_inflight=2, max_batch_clips=4) as srv:
        a = [srv.submit(y, **g) for y, g in reqs]
        b = [srv.submit_borrowed(v, **g) for v, (_, g) in zip(views, reqs)]
        c = srv.submit_borrowed_many(views, [g for _, g in reqs])
        ra = [srv.result(i) for i in a]
        rb = [srv.result(i) for i in b]
        rc = [srv.result(i) for i in c]
    for x, y, z in zip(ra, rb, rc):
        np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(x, z)


def test_without_pinned_pool_room_results_are_unchanged():
    """With a pinned pool too small for anything (1 MiB, below one pool
    chunk), requests wait in pageable copies and batch results come back
    through the slot's staging instead of pool blocks: the results are
    bitwise those of a default server."""
    reqs = _requests(10, seed=11)
    with M.Server(max_inflight=2, max_batch_clips=4) as srv:
        ref = [srv.result(i) for i in [srv.submit(y, **g) for y, g in reqs]]
    with M.Server(max_inflight=2, max_batch_clips=4, host_pinned_bytes=1 << 20) as srv:
        got = [srv.result(i) for i in [srv.submit(y, **g) for y, g in reqs]]
    for x, y in zip(ref, got):
        np.testing.assert_array_equal(x, y)


def test_two_waiters_on_one_request():
    """Two callers wait on the same request: one gets the result, the other
    an invalid-request error (the request is gone once taken), and neither
    waits on after the result is taken."""
    y, g = _requests(1, seed=13)[0]
    outcomes = []
    with M.Server(max_inflight=1, max_batch_clips=1) as srv:
        rid = srv.submit(y, **g)

        def take():
            try:
                outcomes.append(("ok", srv.result(rid, timeout_ms=20000)))
            except RuntimeError as e:
                outcomes.append(("err", str(e)))

        ts = [threading.Thread(target=take) for _ in range(2)]
        for t in ts:
            t.start()
        for t in ts:
            t.join(30)
        assert not any(t.is_alive() for t in ts)
    assert sorted(k for k, _ in outcomes) == ["err", "ok"]
    res = next(v for k, v in outcomes if k == "ok")
    assert O.mfcc_rel_error(res, _oracle(y, g)) < MFCC_TOL
