"""Batched MFCC over many clips (additive API, no counterpart in MetalMom).

``mfcc_batch`` is one call over clips of any lengths.  ``Plan`` keeps a fixed
batch (parameters + clip lengths) resident on the device with its launches
captured in a CUDA graph; inputs and outputs live in device buffers whose
addresses and per-clip offsets the plan exposes.
"""

import numpy as np

from ._bridge import take_buffer
from ._native import ffi, lib


def frontend_params(sr=22050, n_fft=2048, hop_length=None, win_length=None, center=True,
                    pad_mode="constant", n_mels=128, n_mfcc=20, fmin=0.0, fmax=None,
                    top_db=80.0, dft="fft"):
    """An ``MMFrontEndParams`` struct (sentinels: None -> reference defaults)."""
    p = ffi.new("MMFrontEndParams*")
    p.sample_rate = sr
    p.n_fft = n_fft
    p.hop_length = hop_length if hop_length is not None else 0
    p.win_length = win_length if win_length is not None else 0
    p.center = 1 if center else 0
    p.pad_mode = {"constant": lib.MM_PAD_CONSTANT, "reflect": lib.MM_PAD_REFLECT}[pad_mode]
    p.n_mels = n_mels
    p.n_mfcc = n_mfcc
    p.f_min = fmin
    p.f_max = float(fmax) if fmax is not None else 0.0
    p.top_db = float(top_db) if top_db is not None else 0.0
    p.dft_form = {"fft": lib.MM_DFT_FFT_F32, "bf16x3": lib.MM_DFT_GEMM_BF16X3,
                  "bf16": lib.MM_DFT_GEMM_BF16, "f16x3": lib.MM_DFT_GEMM_F16X3}[dft]
    return p


def autotune(clip_samples=661500, n_clips=32, reps=10, **params):
    """Time every launch variant of the frame kernel for these parameters on
    synthetic clips, keep the fastest for this n_fft (process-wide) and return
    {"best": v, "ms": {variant: ms}}."""
    p = frontend_params(**params)
    ms = ffi.new("float[6]")
    best = ffi.new("int32_t*")
    ctx = lib.mm_init()
    try:
        st = lib.mm_autotune(ctx, p, clip_samples, n_clips, reps, ms, best)
        if st != 0:
            raise RuntimeError(f"mm_autotune failed with status {st}")
    finally:
        lib.mm_destroy(ctx)
    return {"best": int(best[0]), "ms": {i: float(ms[i]) for i in range(6) if ms[i] > 0}}


def tune_set(n_fft, variant):
    st = lib.mm_tune_set(n_fft, variant)
    if st != 0:
        raise RuntimeError(f"mm_tune_set failed with status {st}")


def tune_get(n_fft):
    return int(lib.mm_tune_get(n_fft))


def mfcc_batch(clips, **params):
    """MFCC of every clip in one batched launch sequence; returns a list of arrays."""
    clips = [np.ascontiguousarray(c, dtype=np.float32) for c in clips]
    n = len(clips)
    if n == 0:
        return []
    p = frontend_params(**params)
    ptrs = ffi.new("const float*[]", [ffi.cast("const float*", c.ctypes.data) for c in clips])
    lens = ffi.new("int64_t[]", [len(c) for c in clips])
    outs = ffi.new("MMBuffer[]", n)
    ctx = lib.mm_init()
    try:
        status = lib.mm_mfcc_batch(ctx, ptrs, lens, n, p, outs)
        if status != 0:
            raise RuntimeError(f"mm_mfcc_batch failed with status {status}")
        return [take_buffer(outs + i) for i in range(n)]
    finally:
        lib.mm_destroy(ctx)


class Plan:
    """A resident, graph-captured batch of fixed clip lengths.

    ``Plan(lengths, **params)``: one parameter set for every clip.
    ``Plan(lengths, clip_params=[dict, ...], max_clips_per_branch=k)``: each
    clip with its own parameters; clips are grouped by parameter set and the
    groups (cut into branches of at most k clips) run as concurrent branches
    of one graph.
    """

    def __init__(self, lengths, clip_params=None, max_clips_per_branch=0, **params):
        self.lengths = [int(x) for x in lengths]
        self._ctx = lib.mm_init()
        st = ffi.new("int32_t*")
        lens = ffi.new("int64_t[]", self.lengths)
        if clip_params is None:
            self._params = frontend_params(**params)
            self._plan = lib.mm_plan_create(self._ctx, self._params, lens, len(self.lengths), st)
        else:
            if len(clip_params) != len(self.lengths):
                lib.mm_destroy(self._ctx)
                raise ValueError("one parameter dict per clip")
            self._params = ffi.new("MMFrontEndParams[]", len(clip_params))
            for i, kw in enumerate(clip_params):
                self._params[i] = frontend_params(**kw)[0]
            self._plan = lib.mm_plan_create_groups(self._ctx, self._params, lens, len(self.lengths),
                                                   int(max_clips_per_branch), st)
        if self._plan == ffi.NULL:
            lib.mm_destroy(self._ctx)
            raise RuntimeError(f"mm_plan_create failed with status {st[0]}")
        self.n = len(self.lengths)
        self.rows = lib.mm_plan_rows(self._plan)
        self.clip_rows = [lib.mm_plan_clip_rows(self._plan, i) for i in range(self.n)]
        self.branches = lib.mm_plan_branches(self._plan)
        self.frames = [lib.mm_plan_clip_frames(self._plan, i) for i in range(self.n)]
        self.in_offsets = [lib.mm_plan_input_offset(self._plan, i) for i in range(self.n)]
        self.out_offsets = [lib.mm_plan_output_offset(self._plan, i) for i in range(self.n)]
        self.total_frames = lib.mm_plan_total_frames(self._plan)
        self.kernel_launches = lib.mm_plan_kernel_launches(self._plan)

    @property
    def device_input(self) -> int:
        return int(ffi.cast("uintptr_t", lib.mm_plan_device_input(self._plan)))

    @property
    def device_output(self) -> int:
        return int(ffi.cast("uintptr_t", lib.mm_plan_device_output(self._plan)))

    @property
    def device_mel_db(self) -> int:
        return int(ffi.cast("uintptr_t", lib.mm_plan_device_mel_db(self._plan)))

    def clip_mel_db_ptr(self, clip: int) -> int:
        """Device address of clip ``clip``'s frame-major log-mel rows (before
        the top_db floor) of the last execution."""
        p = lib.mm_plan_clip_mel_db(self._plan, clip)
        if p == ffi.NULL:
            raise RuntimeError("no log-mel rows for this clip")
        return int(ffi.cast("uintptr_t", p))

    def clip_max_db(self, clip: int) -> float:
        v = ffi.new("float*")
        st = lib.mm_plan_clip_max_db(self._plan, clip, v)
        if st != 0:
            raise RuntimeError(f"mm_plan_clip_max_db failed with status {st}")
        return float(v[0])

    def execute(self, stream: int = 0):
        st = lib.mm_plan_execute(self._plan, ffi.cast("void*", stream))
        if st != 0:
            raise RuntimeError(f"mm_plan_execute failed with status {st}")

    def execute_timed(self, slot: int, stream: int = 0):
        st = lib.mm_plan_execute_timed(self._plan, ffi.cast("void*", stream), slot)
        if st != 0:
            raise RuntimeError(f"mm_plan_execute_timed failed with status {st}")

    def stage_ms(self, slot: int):
        ms = ffi.new("float[3]")
        st = lib.mm_plan_stage_ms(self._plan, slot, ms)
        if st != 0:
            raise RuntimeError(f"mm_plan_stage_ms failed with status {st}")
        return [ms[0], ms[1], ms[2]]

    def alloc_outputs(self):
        return [np.empty((r, f), dtype=np.float32) for r, f in zip(self.clip_rows, self.frames)]

    def execute_host(self, clips, outs=None, stream: int = 0):
        """Copy ``clips`` in, run, copy MFCCs out (into ``outs`` if given)."""
        clips = [np.ascontiguousarray(c, dtype=np.float32) for c in clips]
        if len(clips) != self.n or any(len(c) != L for c, L in zip(clips, self.lengths)):
            raise ValueError("clips do not match the plan's lengths")
        if outs is None:
            outs = self.alloc_outputs()
        ins = ffi.new("const float*[]", [ffi.cast("const float*", c.ctypes.data) for c in clips])
        ops = ffi.new("float*[]", [ffi.cast("float*", o.ctypes.data) for o in outs])
        st = lib.mm_plan_execute_host(self._plan, ins, ops, ffi.cast("void*", stream))
        if st != 0:
            raise RuntimeError(f"mm_plan_execute_host failed with status {st}")
        return outs

    def close(self):
        if getattr(self, "_plan", None) is not None and self._plan != ffi.NULL:
            lib.mm_plan_destroy(self._plan)
            lib.mm_destroy(self._ctx)
        self._plan = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
