"""Benchmark: audio-hours/s of STFT -> mel -> MFCC on B200.

Workload (default): 256 clips x 30 s at 22050 Hz (661500 samples each) of
seeded synthetic music-like audio; n_fft 2048, hop 512, Hann, centred with
zero padding, 128 Slaney mels (0-11025 Hz), power_to_db(ref 1, amin 1e-10,
top_db 80), 20 MFCC (DCT-II ortho).  One step = the whole batch through the
batched plan.  Inputs (677 MB per GPU) exceed the 126 MB L2, so no flush is
needed between steps.

  value    device-resident throughput (inputs already in HBM), CUDA events
           around the K timed steps on the launching stream, max over ranks;
  e2e      the same metric through the public plan API with pinned host
           buffers: H2D of every clip + kernels + D2H of every MFCC per step;
  roofline dominant kernel (the frame kernel) against measured HBM bandwidth:
           algorithmic bytes = 4*L (audio read) + 4*n_mels*T (log-mel write)
           per clip, divided by its in-region CUDA-event duration;
  cpu_baseline  two CPU stand-ins for the reference's CPU path on a bounded
           sample of the same clips, all host cores: the float32 C port of its
           per-clip algorithm and a NumPy/SciPy (pocketfft) restatement of
           librosa, its parity oracle; the faster one is the value.

`--impl reference` times the faster of those two ports (the reference's own
Swift + Accelerate path cannot be built on Linux) on bounded samples of the
same workload and prints the same JSON line with "impl": "reference"; it loads
no GPU code.
Multi-GPU (torchrun): every rank processes its own 256 clips (weak scaling);
no collective touches the data path.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "audio-hours/sec STFT->mel->MFCC at <=1e-3 dB vs FP64"
UNIT = "audio-hours/s"
SR, N_FFT, HOP, N_MELS, N_MFCC = 22050, 2048, 512, 128, 20
CLIP_SAMPLES = 661500
N_CLIPS = 256


def copy_probe(h2d_bytes, d2h_bytes, stream, chunk, reps=3):
    """Plain pinned-host <-> device copies of the end-to-end leg's bytes (one
    contiguous buffer each way, CUDA events): the PCIe bound of the e2e number."""
    import torch
    src = torch.empty(h2d_bytes // 4, dtype=torch.float32).pin_memory()
    dst = torch.empty(h2d_bytes // 4, dtype=torch.float32, device="cuda")
    back = torch.empty(d2h_bytes // 4, dtype=torch.float32).pin_memory()
    res = {}
    with torch.cuda.stream(stream):
        chunks = [(dst[i:i + chunk // 4], src[i:i + chunk // 4]) for i in range(0, h2d_bytes // 4, chunk // 4)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for a, b in chunks:
            a.copy_(b, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        res["h2d_per_clip_copies_gbs"] = h2d_bytes / (e0.elapsed_time(e1) / 1e3) / 1e9
        for name, a, b, n in (("h2d", dst, src, h2d_bytes), ("d2h", back, dst[: d2h_bytes // 4], d2h_bytes)):
            a.copy_(b, non_blocking=True)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                a.copy_(b, non_blocking=True)
            e1.record(stream)
            torch.cuda.synchronize()
            res[name + "_gbs"] = n * reps / (e0.elapsed_time(e1) / 1e3) / 1e9
    del src, dst, back
    res["bound_s"] = h2d_bytes / (res["h2d_gbs"] * 1e9) + d2h_bytes / (res["d2h_gbs"] * 1e9)
    res["what"] = ("one pinned H2D copy of the step's input bytes plus one D2H copy of its output bytes, "
                   "back to back; bound_value = audio-hours per step / their summed time")
    return res


def workload_config(n_clips):
    return {
        "workload": f"{n_clips} clips x 30 s @22050 Hz, n_fft 2048, hop 512, 128 mels, 20 MFCC",
        "n_clips": n_clips, "clip_samples": CLIP_SAMPLES, "sample_rate": SR, "n_fft": N_FFT,
        "hop_length": HOP, "n_mels": N_MELS, "n_mfcc": N_MFCC, "center": True,
        "pad_mode": "constant", "top_db": 80.0,
        "l2": "inputs 677 MB per GPU > 126 MB L2 (no flush needed)",
    }


def make_clips(n, seed0):
    from metalmom_b200 import synth
    return [synth.music_clip(CLIP_SAMPLES, SR, seed0 + i) for i in range(n)]


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples while a region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


CPU_PORTS = {
    "refcpu": "float32 C port of the reference's per-clip CPU algorithm (radix-2 FFT, dense mel GEMM), "
              "one clip per thread",
    "librosa_port": "NumPy/SciPy restatement of librosa's MFCC (pocketfft rfft, BLAS mel product, scipy DCT), "
                    "float32, one clip per thread",
}


def steady_allocator():
    """glibc malloc in the state a long-running process reaches by itself
    after its first large frees: blocks up to 32 MB from the heap and freed
    memory kept.  A fresh process otherwise maps and unmaps the CPU ports'
    per-clip arrays on every call and spends about half of its time in page
    faults (measured on the B200 hosts' 16 cores: 3.5 audio-h/s for the NumPy
    port in a fresh process against 6.4 in a warm one).  True when set."""
    import ctypes
    try:
        libc = ctypes.CDLL("libc.so.6")
    except OSError:
        return False
    M_TRIM_THRESHOLD, M_MMAP_THRESHOLD = -1, -3
    ok = libc.mallopt(M_MMAP_THRESHOLD, 32 << 20) == 1
    return bool(libc.mallopt(M_TRIM_THRESHOLD, 1 << 30) == 1 and ok)


def cpu_port(name):
    """The MFCC-of-a-clip-list function of one CPU port, all host threads."""
    if name == "refcpu":
        from oracle import refcpu
        return lambda clips: refcpu.mfcc_batch(clips, sr=SR, n_fft=N_FFT, hop=HOP, n_mels=N_MELS,
                                               n_mfcc=N_MFCC, n_threads=os.cpu_count() or 1)
    from oracle import librosa_port
    return lambda clips: librosa_port.mfcc_batch(clips, sr=SR, n_fft=N_FFT, hop=HOP, n_mels=N_MELS,
                                                 n_mfcc=N_MFCC, workers=os.cpu_count() or 1)


def time_cpu_ports(sample):
    """Seconds for `sample` through each CPU port (after one warm-up call on
    one clip per thread); the faster port first."""
    threads = os.cpu_count() or 1
    out = {}
    for name in CPU_PORTS:
        fn = cpu_port(name)
        fn(sample[:min(len(sample), threads)])
        t0 = time.perf_counter()
        fn(sample)
        out[name] = time.perf_counter() - t0
    return dict(sorted(out.items(), key=lambda kv: kv[1]))


def cpu_baseline(clips, n_sample):
    """Both CPU ports timed on the same bounded sample with all host cores;
    the faster one is the reported baseline."""
    sample = clips[:n_sample]
    threads = os.cpu_count() or 1
    steady = steady_allocator()
    secs = time_cpu_ports(sample)
    hours = len(sample) * CLIP_SAMPLES / SR / 3600.0
    best = next(iter(secs))
    return {"value": hours / secs[best], "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(sample)} of the {len(clips)} clips (30 s each); the faster of two CPU ports: "
                      f"{best} ({CPU_PORTS[best]})",
            "seconds": secs[best], "allocator": "steady (mallopt)" if steady else "default",
            "ports": {k: {"audio_hours_per_s": hours / v, "seconds": v, "what": CPU_PORTS[k]}
                      for k, v in secs.items()}}


class _DevView:
    """A float32 device range as a torch tensor (no copy) via __cuda_array_interface__."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 2}


def _device_floats(ptr, n):
    import torch
    return torch.as_tensor(_DevView(ptr, n), device="cuda").cpu().numpy().copy()


def oracle_errors(y, g, mfcc_out, mel_rows=None, clip_max_db=None):
    """Errors of one clip's result against the FP64 oracle: MFCC as max |err|
    / max |c|, and (given the clip's frame-major log-mel rows and maximum)
    mel-dB after the top_db floor, overall, within 60 dB of the maximum, and
    60-80 dB below it beside the reference's own float32 path (the C port)
    on the same values: the bar there is max(1e-3 dB, 2 x the reference's
    error), as in the GPU tests."""
    from oracle import oracle as O, refcpu
    sr, n_fft = g["sr"], g["n_fft"]
    hop, win = g.get("hop_length") or n_fft // 4, g.get("win_length") or n_fft
    n_mels, n_mfcc = g.get("n_mels", 128), g.get("n_mfcc", 20)
    exp_db = O.mel_db(y, sr, n_fft, hop, win, True, n_mels, g.get("fmin", 0.0), g.get("fmax"))
    exp_c = O.dct_basis(min(n_mfcc, n_mels), n_mels) @ exp_db
    out = {"mfcc": O.mfcc_rel_error(np.asarray(mfcc_out).reshape(exp_c.shape), exp_c)}
    if mel_rows is not None:
        T = exp_db.shape[1]
        mel = np.maximum(np.asarray(mel_rows, np.float64).reshape(T, n_mels).T, clip_max_db - 80.0)
        err = np.abs(mel - exp_db)
        near = exp_db >= exp_db.max() - 60.0
        out["mel_db"] = float(err.max())
        out["mel_db_within_60db"] = float(err[near].max())
        far = ~near
        if far.any():
            _, ref_db = refcpu.mfcc(y, sr, n_mfcc, n_fft, hop, win, n_mels, g.get("fmin", 0.0),
                                    g.get("fmax") or 0.0, True, want_mel_db=True)
            err_ref = np.abs(np.asarray(ref_db, np.float64) - exp_db)
            out["mel_db_60_80db"] = float(err[far].max())
            out["reference_f32_mel_db_60_80db"] = float(err_ref[far].max())
    return out


def merge_errors(errs, what):
    """Per-leg maxima of oracle_errors results."""
    out = {"clips_checked": len(errs), "what": what, "oracle": "float64 NumPy restatement",
           "mfcc_max_err_rel_to_max": max(e["mfcc"] for e in errs)}
    if any("mel_db" in e for e in errs):
        out["mel_db_max_abs_err_db"] = max(e["mel_db"] for e in errs if "mel_db" in e)
        out["mel_db_max_abs_err_db_within_60db"] = max(e["mel_db_within_60db"] for e in errs if "mel_db" in e)
    far = [e for e in errs if "mel_db_60_80db" in e]
    if far:
        out["mel_db_60_80db"] = {
            "max_abs_err_db": max(e["mel_db_60_80db"] for e in far),
            "reference_f32_max_abs_err_db": max(e["reference_f32_mel_db_60_80db"] for e in far),
            "within_bar": all(e["mel_db_60_80db"] <= max(1e-3, 2.0 * e["reference_f32_mel_db_60_80db"])
                              for e in far),
            "bar": "per clip: max(1e-3 dB, 2 x the reference float32 path's error on the same values)"}
    return out


def bench_accuracy(plan, clips, n_check=16):
    """The bench run's own outputs (log-mel rows and MFCC, read back from the
    device after the timed region) of `n_check` clips spread over the batch,
    against the FP64 oracle."""
    g = dict(sr=SR, n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS, n_mfcc=N_MFCC)
    idx = sorted({int(round(i * (len(clips) - 1) / max(n_check - 1, 1))) for i in range(n_check)})
    errs = []
    for i in idx:
        T = plan.frames[i]
        mel = _device_floats(plan.clip_mel_db_ptr(i), T * N_MELS)
        got = _device_floats(plan.device_output + 4 * plan.out_offsets[i], N_MFCC * T)
        errs.append(oracle_errors(clips[i], g, got, mel, plan.clip_max_db(i)))
    return merge_errors(errs, f"{len(idx)} of the {len(clips)} bench clips, spread over the batch")


def baseline_leg(plan, clips, world, args):
    """The checker and the CPU baseline (rank 0): FP64 check of this run's own
    mel-dB / MFCC output on 16 clips, then the CPU ports timed at N=1."""
    out = {"accuracy": {"bench": bench_accuracy(plan, clips)}}
    if world == 1:
        out["cpu_baseline"] = cpu_baseline(clips, args.cpu_clips)
    return out


# ---------------------------------------------------------------------------
# served stream: Poisson arrivals, log-normal clip lengths (median 8 s,
# sigma 1, clipped to 0.5-300 s), parameter group drawn uniformly from the
# single-clip music front end, the uneven-batch groups and the speech front
# end; 40 GB admission budget
# ---------------------------------------------------------------------------
SERVE_MUSIC = dict(sr=22050, n_fft=2048, hop_length=512, n_mels=128, n_mfcc=20)
SERVE_SPEECH = dict(sr=16000, n_fft=512, hop_length=160, win_length=400, n_mels=80, n_mfcc=13,
                    fmin=20.0, fmax=8000.0)


def serve_group(rng):
    k = int(rng.integers(3))
    if k == 0:
        return SERVE_MUSIC
    if k == 2:
        return SERVE_SPEECH
    n_fft = int(rng.choice([1024, 2048, 4096]))
    return dict(sr=int(rng.choice([22050, 44100])), n_fft=n_fft, hop_length=n_fft // 4,
                n_mels=int(rng.choice([64, 128])), n_mfcc=20)


def serve_pools():
    from metalmom_b200 import synth
    return {22050: synth.music_clip(300 * 22050, 22050, seed=71),
            44100: synth.music_clip(300 * 44100, 44100, seed=72),
            16000: synth.speech_clip(300 * 16000, 16000, seed=73)}


def serve_requests(pools, rate, duration, seed):
    """(arrival time, clip, params) of a Poisson stream; clips are windows of
    long seeded clips."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        g = serve_group(rng)
        secs = float(np.clip(rng.lognormal(np.log(8.0), 1.0), 0.5, 300.0))
        pool = pools[g["sr"]]
        n = int(secs * g["sr"])
        start = int(rng.integers(0, len(pool) - n + 1))
        out.append((t, pool[start:start + n], g))


def pin_requests(reqs):
    """Each request's samples copied into one pinned host buffer (views)."""
    import torch
    total = sum(len(y) for _, y, _ in reqs)
    buf = torch.empty(total, dtype=torch.float32).pin_memory().numpy()
    views, off = [], 0
    for _, y, _ in reqs:
        v = buf[off:off + len(y)]
        v[:] = y
        views.append(v)
        off += len(y)
    return views


def _pcts(lat_ms):
    lat = np.sort(np.asarray(lat_ms))
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


def serving_leg(duration=3.0, rates=(50, 500, 2000), burst=2000, plain_s=2.0, n_check=32):
    """Continuous batching (Server) on open-loop Poisson streams, a burst for
    the sustained rate, and the plain per-request form (mm_mfcc per request,
    in arrival order) on the same kind of stream."""
    import metalmom_b200 as M
    pools = serve_pools()
    res = {"workload": "Poisson arrivals; lengths log-normal (median 8 s, sigma 1) in 0.5-300 s; "
                       "group uniform over {30 s-clip music front end, uneven-batch groups "
                       "(sr 22050/44100, n_fft 1024/2048/4096, 64/128 mels), speech front end "
                       "(16 kHz, n_fft 512, win 400, hop 160, 80 mels, 13 MFCC)}",
           "budget_bytes": 40 << 30, "streams": []}
    checked = []
    with M.Server(budget_bytes=40 << 30, max_batch_clips=256, max_inflight=4) as srv:
        # one request per parameter group first: tables are built once per group
        groups = [SERVE_MUSIC, SERVE_SPEECH] + [
            dict(sr=sr, n_fft=nf, hop_length=nf // 4, n_mels=nm, n_mfcc=20)
            for sr in (22050, 44100) for nf in (1024, 2048, 4096) for nm in (64, 128)]
        for rid in [srv.submit(pools[g["sr"]][:5 * g["sr"]], **g) for g in groups]:
            srv.result(rid)
        warm = serve_requests(pools, 200, 0.5, seed=9)
        for rid in [srv.submit(y, **g) for _, y, g in warm]:
            srv.result(rid)
        for rate in rates:
            reqs = serve_requests(pools, rate, duration, seed=rate)
            srv.reset_stats()
            t0 = time.perf_counter()
            ids = []
            for t, y, g in reqs:
                while time.perf_counter() - t0 < t:
                    dt = t - (time.perf_counter() - t0)
                    if dt > 0.002:
                        time.sleep(dt - 0.001)
                ids.append(srv.submit(y, **g))
            results = [srv.result(rid) for rid in ids]
            wall = time.perf_counter() - t0
            st = srv.stats()
            checked.extend((y, g, r) for (_, y, g), r in zip(reqs[:n_check], results[:n_check]))
            res["streams"].append({
                "rate_req_s": rate, "requests": len(reqs), "p50_ms": st["latency_p50_ms"],
                "p99_ms": st["latency_p99_ms"], "max_ms": st["latency_max_ms"],
                "audio_hours_per_s": st["audio_seconds_completed"] / 3600.0 / wall,
                "batches": st["batches_launched"], "failed": st["failed"],
                "peak_device_bytes": st["peak_bytes_in_use"]})
        reqs = serve_requests(pools, burst / 0.001, 1.0, seed=4242)[:burst]
        srv.reset_stats()
        t0 = time.perf_counter()
        ids = [srv.submit(y, **g) for _, y, g in reqs]
        for rid in ids:
            srv.result(rid)
        wall = time.perf_counter() - t0
        st = srv.stats()
        res["burst"] = {"requests": len(reqs), "audio_hours_per_s": st["audio_seconds_completed"] / 3600.0 / wall,
                        "p50_ms": st["latency_p50_ms"], "p99_ms": st["latency_p99_ms"],
                        "batches": st["batches_launched"],
                        "client": "one Python thread, mm_server_submit (copies every request into pinned memory)"}
        # saturation: the same requests from a caller's pinned buffers, submitted
        # without a copy (mm_server_submit_borrowed), so the client is not the bound
        pinned = pin_requests(reqs)
        groups = [g for _, _, g in reqs]
        for _ in range(2):
            srv.reset_stats()
            t0 = time.perf_counter()
            ids = srv.submit_borrowed_many(pinned, groups)
            t_sub = time.perf_counter() - t0
            for rid in ids:
                srv.result(rid)
            wall = time.perf_counter() - t0
        st = srv.stats()
        audio_s = st["audio_seconds_completed"]
        res["saturation"] = {"requests": len(reqs), "audio_hours_per_s": audio_s / 3600.0 / wall, "wall_s": wall,
                             "p50_ms": st["latency_p50_ms"], "p99_ms": st["latency_p99_ms"],
                             "batches": st["batches_launched"], "h2d_bytes": int(sum(y.nbytes for y in pinned)),
                             "submit_s": t_sub, "scheduler_launch_ms": st["scheduler_launch_ms"],
                             "scheduler_finish_ms": st["scheduler_finish_ms"],
                             "client": "mm_server_submit_borrowed_many: all requests from pinned host buffers in one call"}
    # the plain per-request form at its own saturation: mm_mfcc per request,
    # back to back, on the same requests
    for _, y, g in reqs[:3]:
        M.mfcc(y, **g)
    t0 = time.perf_counter()
    for _, y, g in reqs:
        M.mfcc(y, **g)
    wall = time.perf_counter() - t0
    res["plain_saturation"] = {"requests": len(reqs), "audio_hours_per_s": audio_s / 3600.0 / wall, "wall_s": wall,
                               "api": "mm_mfcc per request, back to back (host in/out)"}
    res["served_vs_plain_at_saturation"] = res["saturation"]["audio_hours_per_s"] / res["plain_saturation"][
        "audio_hours_per_s"]
    # the plain per-request form on a stream it can follow
    rate = 50
    reqs = serve_requests(pools, rate, plain_s, seed=77)
    for _, y, g in reqs[:3]:
        M.mfcc(y, **g)
    lat, audio = [], 0.0
    t0 = time.perf_counter()
    for t, y, g in reqs:
        while time.perf_counter() - t0 < t:
            time.sleep(0.0002)
        M.mfcc(y, **g)
        lat.append((time.perf_counter() - t0 - t) * 1e3)
        audio += len(y) / g["sr"]
    wall = time.perf_counter() - t0
    p50, p99 = _pcts(lat)
    res["plain_per_request"] = {"rate_req_s": rate, "requests": len(reqs), "p50_ms": p50, "p99_ms": p99,
                                "audio_hours_per_s": audio / 3600.0 / wall,
                                "api": "mm_mfcc per request in arrival order (host in/out)"}
    ab = [s for s in res["streams"] if s["rate_req_s"] == rate]
    if ab:
        res["plain_vs_server_p99"] = p99 / ab[0]["p99_ms"] if ab[0]["p99_ms"] > 0 else None
    # the first n_check served results of every rate against the FP64 oracle
    # (after the streams; MFCC is what a request returns)
    res["accuracy"] = merge_errors([oracle_errors(y, g, r) for y, g, r in checked],
                                   f"the first {n_check} served results of each of the {len(rates)} streams")
    return res


def uneven_workload(n_clips=1024, seed=2024):
    """The uneven batch's clips without their audio: per clip (group params,
    start offset, samples), drawn from one seeded generator, the same on
    every rank."""
    rng = np.random.default_rng(seed)
    work = []
    for _ in range(n_clips):
        n_fft = int(rng.choice([1024, 2048, 4096]))
        g = dict(sr=int(rng.choice([22050, 44100])), n_fft=n_fft, hop_length=n_fft // 4,
                 n_mels=int(rng.choice([64, 128])), n_mfcc=20)
        n = int(rng.uniform(1.0, 120.0) * g["sr"])
        start = int(rng.integers(0, 120 * g["sr"] - n + 1))
        work.append((g, start, n))
    return work


def uneven_shard(work, rank, world):
    """This rank's clip indices: `balanced_shards` over the clips' device cost
    (frames x per-frame cost of their group), in workload order."""
    from metalmom_b200.shard import balanced_shards
    shards = balanced_shards([n for _, _, n in work], world, [g for g, _, _ in work])
    return sorted(shards[rank])


def uneven_leg(stream, rank=0, world=1, dist=None, steps=20, n_clips=1024, seed=2024, variant=None):
    """The uneven batch: 1024 clips, lengths uniform in 1-120 s, each clip
    with its own group (sr 22050/44100, n_fft 1024/2048/4096 with hop n_fft/4,
    64/128 mels, 20 MFCC); launch variants autotuned per n_fft; one grouped
    plan (a graph of concurrent persistent launches, one branch per group),
    inputs resident, CUDA events around `steps` graph replays.  With several
    ranks the clips are routed by device cost (`uneven_shard`), each rank
    runs its own plan, and the time is the max over ranks.  `variant`: one
    fixed launch variant for every n_fft instead of the autotuner (profiling
    runs, where the tuner's timings are distorted)."""
    import torch
    import metalmom_b200 as M
    from metalmom_b200 import synth
    from metalmom_b200.shard import clip_cost, frames_of, max_over_ranks
    pools = {sr: synth.music_clip(120 * sr, sr, seed=sr) for sr in (22050, 44100)}
    work = uneven_workload(n_clips, seed)
    mine = uneven_shard(work, rank, world)
    all_hours = sum(n / g["sr"] for g, _, n in work) / 3600.0
    costs = [sum(clip_cost(work[i][2], **work[i][0]) for i in uneven_shard(work, r, world)) for r in range(world)]
    params = [work[i][0] for i in mine]
    clips = [pools[work[i][0]["sr"]][work[i][1]:work[i][1] + work[i][2]] for i in mine]
    tuned = {}
    for n_fft in (1024, 2048, 4096):
        if variant is not None:
            M.tune_set(n_fft, variant)
            tuned[n_fft] = variant
        else:
            tuned[n_fft] = M.autotune(clip_samples=30 * 22050, n_clips=32, reps=3, sr=22050, n_fft=n_fft,
                                      hop_length=n_fft // 4, n_mels=128, n_mfcc=20)["best"]
    plan = M.Plan([len(c) for c in clips], clip_params=params)
    sh = stream.cuda_stream
    plan.execute_host(clips, stream=sh)
    for _ in range(3):
        plan.execute(stream=sh)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        plan.execute(stream=sh)
    b.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(b) / steps, dist, device="cuda")
    if rank != 0:
        plan.close()
        return None
    hours = all_hours
    # the longest clip of every group: its MFCC and log-mel rows from the last
    # replay against the FP64 oracle
    res = plan.execute_host(clips, stream=sh)
    torch.cuda.synchronize()
    longest = {}
    for i, g in enumerate(params):
        key = tuple(sorted(g.items()))
        if key not in longest or len(clips[i]) > len(clips[longest[key]]):
            longest[key] = i
    errs = []
    for i in longest.values():
        g = params[i]
        mel = _device_floats(plan.clip_mel_db_ptr(i), plan.frames[i] * g["n_mels"])
        errs.append(oracle_errors(clips[i], g, res[i], mel, plan.clip_max_db(i)))
    out = {"workload": f"{n_clips} clips, lengths U[1,120] s, per-clip group from sr {{22050, 44100}} x "
                       "n_fft {1024, 2048, 4096} (hop n_fft/4) x mels {64, 128}, 20 MFCC",
           "audio_hours": hours, "ms_per_step": ms, "audio_hours_per_s": hours / (ms / 1e3),
           "samples_per_s": sum(n for _, _, n in work) / (ms / 1e3),
           "frames_per_s": sum(frames_of(n, g["n_fft"], g["hop_length"], True) for g, _, n in work) / (ms / 1e3),
           "sharding": ("1 GPU" if world == 1 else
                        f"{world} ranks, clips routed by device cost (balanced_shards), max over ranks; "
                        f"rank cost max / mean {max(costs) / (sum(costs) / world):.3f}"),
           "groups": len({tuple(sorted(g.items())) for g in params}), "branches": plan.branches,
           "gpu_launches_per_step": plan.kernel_launches, "tuned_variant_per_n_fft": tuned,
           "timing": "CUDA events around graph replays, inputs resident (> L2)",
           "accuracy": merge_errors(errs, "the longest clip of each group" +
                                    ("" if world == 1 else " among rank 0's clips"))}
    plan.close()
    return out


def precision_leg(stream, n_clips=512, steps=10):
    """The speech front end (16 kHz, n_fft 512, win 400, hop 160, 80 mels
    20-8000 Hz, 13 MFCC) on 512 clips x 10 s in four DFT forms: the float32
    FFT, the DFT as a tcgen05 GEMM with bf16x3 split products (float32
    accumulation), with plain bf16, and with fp16x3 split products of each
    frame scaled by a power of two; device-resident throughput of each
    (graph replays, CUDA events) and max/mean mel-dB and MFCC error against the
    FP64 oracle on 4 clips."""
    import torch
    import metalmom_b200 as M
    from metalmom_b200 import synth
    from oracle import oracle as O
    pool = synth.speech_clip(600 * 16000, 16000, seed=2025)
    rng = np.random.default_rng(7)
    L = 160000
    starts = rng.integers(0, len(pool) - L, n_clips)
    clips = [pool[s:s + L] for s in starts]
    M.autotune(clip_samples=L, n_clips=32, reps=3, **SERVE_SPEECH)
    sh = stream.cuda_stream
    check = [0, 1, n_clips // 2, n_clips - 1]
    exp_db = [O.mel_db(clips[i], 16000, 512, 160, 400, True, 80, 20.0, 8000.0) for i in check]
    exp_c = [O.mfcc(clips[i], 16000, 13, 512, 160, 400, 80, 20.0, 8000.0) for i in check]
    out = {"workload": f"{n_clips} clips x 10 s @16 kHz speech-like, n_fft 512, win 400, hop 160, 80 mels, 13 MFCC",
           "forms": {}}
    hours = n_clips * L / 16000 / 3600.0
    for form in ("fft", "bf16x3", "bf16", "f16x3"):
        with M.Plan([L] * n_clips, dft=form, **SERVE_SPEECH) as plan:
            res = plan.execute_host(clips, stream=sh)
            for _ in range(3):
                plan.execute(stream=sh)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(steps):
                plan.execute(stream=sh)
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / steps
            frame0 = np.concatenate([[0], np.cumsum(plan.frames)])
            db_max, db_mean, c_max = 0.0, [], 0.0
            for j, i in enumerate(check):
                T = plan.frames[i]
                mel = _device_floats(plan.device_mel_db + 4 * int(frame0[i]) * 80, T * 80)
                mel = np.maximum(mel.reshape(T, 80).T.astype(np.float64), plan.clip_max_db(i) - 80.0)
                d = np.abs(mel - exp_db[j])
                db_max = max(db_max, float(d.max()))
                db_mean.append(float(d.mean()))
                c_max = max(c_max, O.mfcc_rel_error(res[i], exp_c[j]))
        out["forms"][form] = {"audio_hours_per_s": hours / (ms / 1e3), "ms_per_step": ms,
                              "mel_db_max_abs_err_db": db_max, "mel_db_mean_abs_err_db": float(np.mean(db_mean)),
                              "mfcc_max_err_rel_to_max": c_max}
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import metalmom_b200 as M
    from metalmom_b200.shard import max_over_ranks

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    n_clips = args.clips
    clips = make_clips(n_clips, seed0=1000 * rank)
    lengths = [len(c) for c in clips]
    if args.variant is None:
        tune = M.autotune(clip_samples=CLIP_SAMPLES, n_clips=min(n_clips, 64), reps=5, sr=SR,
                          n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS, n_mfcc=N_MFCC)
    else:  # a fixed launch variant (profiling runs, where the tuner's timings are distorted)
        M.tune_set(N_FFT, args.variant)
        tune = {"best": args.variant, "ms": []}
    plan = M.Plan(lengths, sr=SR, n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS, n_mfcc=N_MFCC)
    # an explicit stream: handle 0 (the legacy default stream) would mean "the
    # plan's own stream" to the C ABI, outside these events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    assert sh != 0

    # pinned host buffers for the end-to-end leg, which runs through a plan cut
    # into branches so that one branch's copies overlap another's kernels
    # (one pinned [n_clips, samples] array and one [n_clips, rows, frames]
    # array, passed as per-clip row views, as a caller holding a batch does)
    pin_in = torch.from_numpy(np.stack(clips)).pin_memory()
    in_np = list(pin_in.numpy())
    pin_out = torch.empty((n_clips, plan.rows, plan.frames[0]), dtype=torch.float32).pin_memory()
    out_np = list(pin_out.numpy())
    assert all(f == plan.frames[0] for f in plan.frames)
    plan_io = M.Plan(lengths, clip_params=[dict(sr=SR, n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS,
                                                n_mfcc=N_MFCC)] * n_clips,
                     max_clips_per_branch=args.e2e_branch_clips)
    plan.execute_host(in_np, out_np, stream=sh)  # uploads the inputs once
    torch.cuda.synchronize()

    hours_per_step = n_clips * CLIP_SAMPLES / SR / 3600.0
    K, W = args.steps, args.warmup

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident timed region
    for i in range(W):
        plan.execute_timed(i % 64, stream=sh)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        start.record(stream)
        for i in range(K):
            plan.execute_timed(i % 64, stream=sh)
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end)
    stage = np.array([plan.stage_ms(i) for i in range(min(K, 64))])
    frame_ms = float(stage[:, 1].mean())
    dct_ms = float(stage[:, 2].mean())
    ms = max_over_ranks(ms, dist, device="cuda")
    ms_step = ms / K
    value = hours_per_step * world / (ms_step / 1e3)

    # ---- end-to-end through the public API (pinned host in/out every step)
    for _ in range(max(1, W // 2)):
        plan_io.execute_host(in_np, out_np, stream=sh)
    torch.cuda.synchronize()
    barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ke = max(1, min(K, args.e2e_steps))
    e_start.record(stream)
    for _ in range(ke):
        plan_io.execute_host(in_np, out_np, stream=sh)
    e_end.record(stream)
    torch.cuda.synchronize()
    e_ms = e_start.elapsed_time(e_end)
    e_ms = max_over_ranks(e_ms, dist, device="cuda")
    e2e_value = hours_per_step * world / (e_ms / ke / 1e3)
    h2d = sum(c.nbytes for c in in_np)
    d2h = sum(o.nbytes for o in out_np)
    copy = copy_probe(h2d, d2h, stream, in_np[0].nbytes) if rank == 0 else None

    # ---- the uneven mixed-group batch: every rank, clips routed by device cost
    uneven = None if args.no_uneven else uneven_leg(stream, rank, world, dist, variant=args.variant)

    # ---- the plain one-clip-per-launch GPU form, for comparison
    per_clip = None
    if rank == 0:
        n_pc = min(32, n_clips)  # wall clock over pageable copies: a larger sample steadies it
        for c in clips[:4]:
            M.mfcc(c, sr=SR, n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS, n_mfcc=N_MFCC)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for c in clips[:n_pc]:
            M.mfcc(c, sr=SR, n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS, n_mfcc=N_MFCC)
        torch.cuda.synchronize()
        host_s = time.perf_counter() - t0
        one = M.Plan([CLIP_SAMPLES], sr=SR, n_fft=N_FFT, hop_length=HOP, n_mels=N_MELS, n_mfcc=N_MFCC)
        one.execute_host([clips[0]], stream=sh)
        for _ in range(3):
            one.execute(stream=sh)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_dev = 64
        p0.record(stream)
        for _ in range(n_dev):
            one.execute(stream=sh)
        p1.record(stream)
        torch.cuda.synchronize()
        dev_ms = p0.elapsed_time(p1) / n_dev
        one.close()
        clip_h = CLIP_SAMPLES / SR / 3600.0
        per_clip = {
            "e2e_value": n_pc * clip_h / host_s, "unit": UNIT,
            "e2e_api": f"mm_mfcc per clip (host in/out, context per call), {n_pc} clips, wall clock",
            "device_value": clip_h / (dev_ms / 1e3),
            "device_api": f"single-clip plan replayed {n_dev} times (input resident), CUDA events",
        }

    result = None
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        hbm = peaks.get("hbm_gbs")
        peak_note = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        T_total = plan.total_frames
        alg_bytes = 4.0 * sum(lengths) + 4.0 * N_MELS * T_total
        achieved = alg_bytes / (frame_ms / 1e3) / 1e9
        pipe_bytes = 4.0 * sum(lengths) + 4.0 * N_MFCC * T_total
        flops_fft = 2.5 * N_FFT * np.log2(N_FFT) * T_total
        traffic = None
        warp = tune["best"] == 3
        kname = {3: "frame_warp_kernel<11>", 5: "frame_tc_kernel"}.get(
            tune["best"], f"frontend_kernel<11,V{tune['best']},MELDB>")
        tp = os.path.join(ROOT, "profiles", kname.split("<")[0] + "_256clips_traffic.txt")
        if os.path.exists(tp) and n_clips == N_CLIPS:
            for line in open(tp):
                if line.startswith("bytes_per_launch:"):
                    traffic = float(line.split(":")[1])
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded music-like clips)",
            "config": workload_config(n_clips),
            "sharding": f"clip-sharded x{world}, no collective on the data path" if world > 1 else "1 GPU",
            "roofline": {"bound": "hbm", "kernel": kname,
                         "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": peak_note, "traffic": traffic,
                         "kernel_ms": frame_ms, "dct_ms": dct_ms,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "pipeline_frac": pipe_bytes / (ms_step / 1e3) / 1e9 / hbm,
                         "fp32_fft_tflops": flops_fft / (frame_ms / 1e3) / 1e12,
                         # the kernel's binding roof is compute, not HBM: FFT-form flops
                         # (2.5 N log2 N per frame) against the FP32 CUDA-core peak, nominal
                         # (148 SMs x 128 lanes x 2 flop x the sampled max SM clock)
                         "fp32_peak_tflops_nominal": 148 * 128 * 2 * (peaks.get("sm_max_mhz") or 1965.0) / 1e6,
                         "fp32_fft_frac_of_nominal": flops_fft / (frame_ms / 1e3) / 1e12
                         / (148 * 128 * 2 * (peaks.get("sm_max_mhz") or 1965.0) / 1e6)},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": ke, "branches": plan_io.branches,
                    "api": "Plan.execute_host (mm_plan_execute_host), pinned host buffers",
                    "copy_roofline": dict(copy, bound_value=hours_per_step / copy["bound_s"],
                                          frac=e2e_value / (hours_per_step / copy["bound_s"]))},
            "clocks": clk.summary(),
            "gpu_launches": K * plan.kernel_launches,
            "one_clip_per_launch": per_clip,
            "samples_per_s": world * sum(lengths) / (ms_step / 1e3),
            "frames_per_s": world * T_total / (ms_step / 1e3),
            "batched_vs_one_clip": {"device": value / world / per_clip["device_value"],
                                    "e2e": e2e_value / world / per_clip["e2e_value"]},
            "autotune": {"variant": tune["best"], "variant_ms": tune["ms"],
                         "sample": f"{min(n_clips, 64)} clips of the workload shape"},
        }
        if not args.no_cpu:
            result.update(baseline_leg(plan, clips, world, args))
        if not args.no_serve:
            result["serving"] = serving_leg()
        if uneven is not None:
            result["uneven_batch"] = uneven
        if not args.no_precision:
            result["precision_forms"] = precision_leg(stream)
        # per-leg accuracy against the FP64 oracle, in one place
        acc = result.setdefault("accuracy", {})
        if "uneven_batch" in result:
            acc["uneven_batch"] = result["uneven_batch"]["accuracy"]
        if "serving" in result:
            acc["serving"] = result["serving"]["accuracy"]
        if "precision_forms" in result:
            f = result["precision_forms"]["forms"]["fft"]
            acc["speech_fft"] = {"clips_checked": 4, "mel_db_max_abs_err_db": f["mel_db_max_abs_err_db"],
                                 "mfcc_max_err_rel_to_max": f["mfcc_max_err_rel_to_max"]}
    plan.close()
    plan_io.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_reference(args, rank):
    """The reference arm: MetalMom's CPU path cannot be built on Linux (Swift +
    Apple Accelerate), so this times the faster of its two CPU stand-ins (the
    C port of its per-clip algorithm, and the NumPy/SciPy restatement of
    librosa, its parity oracle) on the host cores.  Loads no GPU code: the
    clips come from the seeded generator module alone."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    n = args.ref_clips
    clips = make_clips(n, seed0=0)
    steady = steady_allocator()
    secs = time_cpu_ports(clips)  # picks the port; not part of the timed steps
    port = next(iter(secs))
    fn = cpu_port(port)
    for _ in range(args.warmup):
        fn(clips)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fn(clips)
        times.append(time.perf_counter() - t0)
    dt = float(np.mean(times))
    hours = n * CLIP_SAMPLES / SR / 3600.0
    v = hours / dt
    sample = (f"{n} of the {N_CLIPS} workload clips per step (30 s each), timed as a rate; "
              f"{port}: {CPU_PORTS[port]}")
    return {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(N_CLIPS), "impl": "reference",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "ports_one_step_s": secs,
                         "allocator": "steady (mallopt)" if steady else "default"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "MetalMom's CPU path is Swift + Apple Accelerate and cannot be built on Linux; this arm times "
                "the faster of its two CPU stand-ins (oracle/refcpu.c, oracle/librosa_port.py) on the host cores.",
    }


def kernel_case(args):
    """One device-resident MFCC plan at another frame size (hop n_fft/4, 128
    mels, 20 MFCC) over --clips 30 s clips at 22050 Hz, --variant fixed, for
    kernel profiles: prints the mean plan time over --steps replays."""
    import torch
    import metalmom_b200 as M
    from metalmom_b200 import synth
    n_fft = args.kernel_case
    base = synth.music_clip(CLIP_SAMPLES + 997 * args.clips, SR, seed=5)
    clips = [base[997 * i: 997 * i + CLIP_SAMPLES] for i in range(args.clips)]
    if args.variant is not None:
        M.tune_set(n_fft, args.variant)
    plan = M.Plan([CLIP_SAMPLES] * args.clips, sr=SR, n_fft=n_fft, hop_length=n_fft // 4, n_mels=N_MELS,
                  n_mfcc=N_MFCC)
    stream = torch.cuda.Stream()
    plan.execute_host(clips, stream=stream.cuda_stream)
    for _ in range(args.warmup):
        plan.execute(stream=stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        plan.execute(stream=stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    out = {"kernel_case": {"n_fft": n_fft, "hop_length": n_fft // 4, "clips": args.clips,
                           "variant": M.tune_get(n_fft), "ms_per_step": a.elapsed_time(b) / max(args.steps, 1)}}
    plan.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--clips", type=int, default=N_CLIPS)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-clips", type=int, default=128)
    # the reference arm's clips per step: as many as the in-bench CPU baseline
    # takes, so that the ports' per-call setup (filterbank and DCT tables,
    # thread pool) is amortised the same way
    ap.add_argument("--ref-clips", type=int, default=128)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--variant", type=int, default=None,
                    help="fixed frame-kernel launch variant for every n_fft (no autotuning)")
    ap.add_argument("--e2e-branch-clips", type=int, default=32)
    ap.add_argument("--kernel-case", type=int, default=None, metavar="N_FFT",
                    help="only a device-resident plan at this n_fft (kernel profiles); no bench line")
    args = ap.parse_args()
    if args.kernel_case is not None:
        print(json.dumps(kernel_case(args)))
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, rank)
    else:
        res = run_ours(args, rank, world, local_rank)
    if rank == 0 and res is not None:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
