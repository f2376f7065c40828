"""Serving front end (additive API, no counterpart in MetalMom).

``Server`` wraps ``mm_server_*``: a native scheduler thread that batches
pending MFCC requests by parameter group (continuous batching), admits
batches against a device-memory budget and runs several of them at once on
separate CUDA streams.  ``submit`` returns a request id immediately;
``result`` / ``poll`` hand back the ``[n_mfcc, n_frames]`` array.
"""

import numpy as np

from ._bridge import take_buffer
from ._native import ffi, lib
from .batch import frontend_params

PENDING = lib.MM_PENDING

STAT_KEYS = ["submitted", "completed", "failed", "pending", "inflight_batches", "batches_launched",
             "bytes_in_use", "peak_bytes_in_use", "audio_seconds_completed", "latency_p50_ms",
             "latency_p99_ms", "latency_mean_ms", "latency_max_ms", "scheduler_launch_ms",
             "scheduler_finish_ms"]


class Server:
    def __init__(self, budget_bytes=40 << 30, max_batch_clips=256, max_inflight=4, host_pinned_bytes=0):
        cfg = ffi.new("MMServerConfig*")
        cfg.device_budget_bytes = int(budget_bytes)
        cfg.max_batch_clips = int(max_batch_clips)
        cfg.max_inflight = int(max_inflight)
        cfg.host_pinned_bytes = int(host_pinned_bytes)
        st = ffi.new("int32_t*")
        self._borrowed = {}
        self._srv = lib.mm_server_create(cfg, st)
        if self._srv == ffi.NULL:
            raise RuntimeError(f"mm_server_create failed with status {st[0]}")

    def submit(self, y, **params) -> int:
        """Queue one clip; ``params`` as ``mfcc_batch`` (sr, n_fft, hop_length, ...)."""
        y = np.ascontiguousarray(y, dtype=np.float32)
        p = frontend_params(**params)
        rid = ffi.new("int64_t*")
        st = lib.mm_server_submit(self._srv, ffi.cast("const float*", y.ctypes.data), len(y), p, rid)
        if st != 0:
            raise RuntimeError(f"mm_server_submit failed with status {st}")
        return int(rid[0])

    def submit_borrowed(self, y, **params) -> int:
        """Queue one clip without copying it: ``y`` (a contiguous float32
        array, ideally in pinned memory) is read in place when its batch
        starts, and is held here until its result is taken."""
        if not (isinstance(y, np.ndarray) and y.dtype == np.float32 and y.flags.c_contiguous):
            raise ValueError("submit_borrowed needs a contiguous float32 array")
        p = frontend_params(**params)
        rid = ffi.new("int64_t*")
        st = lib.mm_server_submit_borrowed(self._srv, ffi.cast("const float*", y.ctypes.data), len(y), p, rid)
        if st != 0:
            raise RuntimeError(f"mm_server_submit_borrowed failed with status {st}")
        self._borrowed[int(rid[0])] = y
        return int(rid[0])

    def submit_borrowed_many(self, clips, params_list) -> list:
        """``submit_borrowed`` for many requests in one native call (the
        client's per-request cost is one cffi argument each)."""
        n = len(clips)
        for y in clips:
            if not (isinstance(y, np.ndarray) and y.dtype == np.float32 and y.flags.c_contiguous):
                raise ValueError("submit_borrowed_many needs contiguous float32 arrays")
        ptrs = ffi.new("const float*[]", [ffi.cast("const float*", y.ctypes.data) for y in clips])
        lens = ffi.new("int64_t[]", [len(y) for y in clips])
        ps = ffi.new("MMFrontEndParams[]", n)
        cache = {}
        for i, kw in enumerate(params_list):
            key = tuple(sorted(kw.items()))
            if key not in cache:
                cache[key] = frontend_params(**kw)[0]
            ps[i] = cache[key]
        ids = ffi.new("int64_t[]", n)
        st = lib.mm_server_submit_borrowed_many(self._srv, ptrs, lens, n, ps, ids)
        out = [int(ids[i]) for i in range(n)]
        for rid, y in zip(out, clips):
            if rid >= 0:
                self._borrowed[rid] = y
        if st != 0:
            raise RuntimeError(f"mm_server_submit_borrowed_many failed with status {st}")
        return out

    def poll(self, rid: int):
        """The result if the request is done, else None."""
        out = ffi.new("MMBuffer*")
        st = lib.mm_server_poll(self._srv, rid, out)
        if st == PENDING:
            return None
        self._borrowed.pop(rid, None)
        if st != 0:
            raise RuntimeError(f"request {rid} failed with status {st}")
        return take_buffer(out)

    def result(self, rid: int, timeout_ms: int = -1):
        """Wait for the request (``timeout_ms`` < 0: no limit) and return its MFCC."""
        out = ffi.new("MMBuffer*")
        st = lib.mm_server_wait(self._srv, rid, int(timeout_ms), out)
        if st == PENDING:
            raise TimeoutError(f"request {rid} not done after {timeout_ms} ms")
        self._borrowed.pop(rid, None)
        if st != 0:
            raise RuntimeError(f"request {rid} failed with status {st}")
        return take_buffer(out)

    def stats(self) -> dict:
        s = ffi.new("MMServerStats*")
        st = lib.mm_server_stats(self._srv, s)
        if st != 0:
            raise RuntimeError(f"mm_server_stats failed with status {st}")
        return {k: getattr(s, k) for k in STAT_KEYS}

    def reset_stats(self):
        lib.mm_server_reset_stats(self._srv)

    def close(self):
        if getattr(self, "_srv", None) is not None and self._srv != ffi.NULL:
            lib.mm_server_destroy(self._srv)
        self._srv = None
        self._borrowed = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
