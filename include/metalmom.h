/*
 * metalmom.h -- C ABI of the B200 spectral front end (libmetalmom.so).
 *
 * The first part is a byte-compatible restatement of the MetalMom bridge
 * header (Sources/MetalMomCBridge/include/metalmom.h in the MetalMom project)
 * for the entry points of the STFT -> mel -> MFCC path.  Callers written
 * against MetalMom (its Python cffi layer, Swift hosts) bind these symbols
 * unchanged.  The second part adds batched, device-resident and serving entry
 * points that have no counterpart in MetalMom.
 *
 * Every compute entry point runs on the CUDA device that is current for the
 * calling thread; there is no CPU fallback.  Without a usable GPU the compute
 * calls return MM_ERR_METAL_UNAVAILABLE (the reference's "no Metal device"
 * code, reused as "no CUDA device").
 */
#ifndef METALMOM_H
#define METALMOM_H

#include <stdint.h>

#if defined(__GNUC__) && defined(MM_BUILDING_LIBRARY)
#define MM_API __attribute__((visibility("default")))
#else
#define MM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (reference metalmom.h:6-11). */
#define MM_OK 0
#define MM_ERR_INVALID_INPUT -1
#define MM_ERR_METAL_UNAVAILABLE -2
#define MM_ERR_ALLOC_FAILED -3
#define MM_ERR_INTERNAL -4

/* Result buffer (reference metalmom.h:14-20): 88 bytes, data malloc'd by the
 * library and released with mm_buffer_free. */
typedef struct {
    float* data;
    int64_t shape[8];
    int32_t ndim;
    int32_t dtype; /* 0 = float32 */
    int64_t count;
} MMBuffer;

/* STFT parameters (reference metalmom.h:23-28). */
typedef struct {
    int32_t n_fft;
    int32_t hop_length;
    int32_t win_length;
    int32_t center; /* 1 = pad n_fft/2 zeros on both sides */
} MMSTFTParams;

/* Opaque context.  Not thread-safe: create one per thread (reference
 * metalmom.h:30-31). */
typedef void* mm_context;

/* ---- Reference entry points ------------------------------------------- */

/* Replaces MetalMomBridge/Bridge.swift:22 (mm_init). */
MM_API mm_context mm_init(void);

/* Replaces Bridge.swift:33 (mm_destroy); destroying twice is a no-op. */
MM_API void mm_destroy(mm_context ctx);

/* Replaces Bridge.swift:44 (mm_stft): magnitude |X|, shape [n_fft/2+1, n_frames].
 * hop_length / win_length are used as given (no sentinels), as in the
 * reference; n_fft must be a power of two.  hop_length <= 0 is rejected with
 * MM_ERR_INVALID_INPUT (the reference divides by it). */
MM_API int32_t mm_stft(mm_context ctx, const float* signal_data, int64_t signal_length,
                int32_t sample_rate, const MMSTFTParams* params, MMBuffer* out);

/* Additive: the C-ABI form of STFT.computeComplex (Spectral/STFT.swift:512-668).
 * X[k] of each zero-centre-padded windowed frame, the imaginary parts of DC and
 * Nyquist set to 0.  out: float32 [n_fft/2+1, n_frames, 2] (interleaved re, im;
 * exactly the stft_data layout mm_istft takes), ndim 3, count 2 * n_freqs *
 * n_frames.  hop_length <= 0 -> n_fft / 4 and win_length <= 0 -> n_fft (the
 * defaults of computeComplex).  A non-power-of-two n_fft or a signal shorter
 * than one frame gives MM_OK with n_frames = 0, as computeComplex returns an
 * empty [n_freqs, 0] signal. */
MM_API int32_t mm_stft_complex(mm_context ctx, const float* signal_data, int64_t signal_length,
                int32_t sample_rate, const MMSTFTParams* params, MMBuffer* out);

/* Replaces Bridge.swift:144 (mm_istft): inverse STFT by overlap-add of the
 * windowed inverse transforms, divided by the overlapped squared windows.
 * stft_data: interleaved complex [n_freqs, n_frames] row-major (stft_count =
 * 2 * n_freqs * n_frames floats); n_fft = 2 * (n_freqs - 1); centre padding
 * trimmed when center != 0; output_length > 0 truncates or zero-pads.
 * Output ndim 1.  hop_length <= 0, n_freqs < 2 or a short stft_count are
 * rejected (MM_ERR_INVALID_INPUT). */
MM_API int32_t mm_istft(mm_context ctx, const float* stft_data, int64_t stft_count,
                        int32_t n_freqs, int32_t n_frames, int32_t sample_rate,
                        int32_t hop_length, int32_t win_length, int32_t center,
                        int64_t output_length, MMBuffer* out);

/* Replaces Bridge.swift:225 (mm_amplitude_to_db): 20*log10(max(x,amin)/ref),
 * floored at max-top_db when top_db > 0.  Output ndim 1, shape [count]. */
MM_API int32_t mm_amplitude_to_db(mm_context ctx, const float* data, int64_t count,
                           float ref, float amin, float top_db, MMBuffer* out);

/* Replaces Bridge.swift:267 (mm_power_to_db): 10*log10(max(x,amin)/ref),
 * floored at max-top_db when top_db > 0.  Output ndim 1, shape [count]. */
MM_API int32_t mm_power_to_db(mm_context ctx, const float* data, int64_t count,
                       float ref, float amin, float top_db, MMBuffer* out);

/* Replaces Bridge.swift:310 (mm_mel_spectrogram): FB @ |X|^power, shape
 * [n_mels, n_frames].  Sentinels: hop<=0 -> n_fft/4, win<=0 -> n_fft,
 * f_max<=0 -> sr/2. */
MM_API int32_t mm_mel_spectrogram(mm_context ctx, const float* signal_data, int64_t signal_length,
                           int32_t sample_rate, int32_t n_fft, int32_t hop_length,
                           int32_t win_length, int32_t center, float power,
                           int32_t n_mels, float f_min, float f_max, MMBuffer* out);

/* Replaces Bridge.swift:402 (mm_mfcc): DCT-II ortho of power_to_db(mel, ref 1,
 * amin 1e-10, top_db 80), shape [min(n_mfcc, n_mels), n_frames]. */
MM_API int32_t mm_mfcc(mm_context ctx, const float* signal_data, int64_t signal_length,
                int32_t sample_rate, int32_t n_mfcc, int32_t n_fft,
                int32_t hop_length, int32_t win_length,
                int32_t n_mels, float f_min, float f_max,
                int32_t center, MMBuffer* out);

/* Replaces Bridge.swift:3695 (mm_buffer_free): frees data, zeroes the struct;
 * NULL-safe. */
MM_API void mm_buffer_free(MMBuffer* buf);

/* ---- Features built on the front end (reference entry points) ---------- */

/* Replaces Bridge.swift:1319 (mm_onset_strength): spectral flux of the
 * power_to_db(top_db 80) mel spectrogram (lag 1), mean over bands (aggregate
 * != 0, shape [1, n_frames]) or per band ([n_mels, n_frames]), shifted by
 * lag + n_fft/(2 hop) when centred.  hop <= 0 -> 512, f_max <= 0 -> sr/2. */
MM_API int32_t mm_onset_strength(mm_context ctx, const float* signal_data, int64_t signal_length,
                                 int32_t sample_rate, int32_t n_fft, int32_t hop_length,
                                 int32_t n_mels, float f_min, float f_max,
                                 int32_t center, int32_t aggregate, MMBuffer* out);

/* Replaces Bridge.swift:934 (mm_delta): Savitzky-Golay derivative of order
 * `order` along time of [n_features, n_frames] (librosa mode 'interp'). */
MM_API int32_t mm_delta(mm_context ctx, const float* data, int64_t count,
                        int32_t n_features, int32_t n_frames,
                        int32_t width, int32_t order, MMBuffer* out);

/* Replaces Bridge.swift:959 (mm_stack_memory): [n_features*n_steps, n_frames]. */
MM_API int32_t mm_stack_memory(mm_context ctx, const float* data, int64_t count,
                               int32_t n_features, int32_t n_frames,
                               int32_t n_steps, int32_t delay, MMBuffer* out);

/* ---- Additive entry points (no counterpart in the reference) ----------- */

/* melspectrogram(S=...) on the GPU (python/metalmom/feature.py:50-57 applies
 * the `_mel_fb.py` filterbank to S with numpy).  S: [n_freqs, n_frames]
 * row-major, n_freqs == n_fft/2 + 1 (else MM_ERR_INVALID_INPUT, where numpy's
 * matmul raises); f_max <= 0 -> sr/2.  out: [n_mels, n_frames]; a frame whose
 * column holds a non-finite value is NaN in every band, as in the dense
 * product. */
MM_API int32_t mm_mel_project(mm_context ctx, const float* S, int64_t count, int32_t n_freqs,
                              int32_t n_frames, int32_t sample_rate, int32_t n_fft, int32_t n_mels,
                              float f_min, float f_max, MMBuffer* out);

/* mfcc(S=...) on the GPU (feature.py:130-134: scipy dct(S, axis=0, type=2,
 * norm='ortho')[:n_mfcc]).  S: [n_rows, n_frames]; out: [min(n_out, n_rows),
 * n_frames].  No top_db floor. */
MM_API int32_t mm_dct_ortho(mm_context ctx, const float* S, int64_t count, int32_t n_rows,
                            int32_t n_frames, int32_t n_out, MMBuffer* out);

/* power_to_db / amplitude_to_db of a DEVICE buffer on the caller's stream
 * (cudaStream_t as void*; asynchronous).  ref_mode 0: divide by `ref`;
 * ref_mode 1: by max(d_in) computed on the device, as ref=np.max
 * (feature.py:247-248), NaN when d_in holds a NaN.  top_db <= 0: no floor.
 * d_out may equal d_in. */
MM_API int32_t mm_power_to_db_device(const float* d_in, int64_t count, float ref, int32_t ref_mode,
                                     float amin, float top_db, float* d_out, void* stream);
MM_API int32_t mm_amplitude_to_db_device(const float* d_in, int64_t count, float ref, int32_t ref_mode,
                                         float amin, float top_db, float* d_out, void* stream);

#define MM_PAD_CONSTANT 0 /* zeros: the reference's centering */
#define MM_PAD_REFLECT 1  /* mirror without repeating the edge sample */

/* How the spectrum is computed: the float32 FFT (default), or the DFT as a
 * GEMM on the tensor cores (n_fft 256..1024, window <= n_fft) with bf16
 * operands split in two parts (three products, float32 accumulation), plain
 * bf16, or fp16 operands split in two parts (three products) after scaling
 * each frame by a power of two.  The GEMM forms exist for the precision
 * comparison. */
#define MM_DFT_FFT_F32 0
#define MM_DFT_GEMM_BF16X3 1
#define MM_DFT_GEMM_BF16 2
#define MM_DFT_GEMM_F16X3 3

/* One front-end parameter group.  Sentinels as in mm_mfcc. */
typedef struct {
    int32_t sample_rate;
    int32_t n_fft;
    int32_t hop_length; /* <= 0: n_fft/4 */
    int32_t win_length; /* <= 0: n_fft */
    int32_t center;
    int32_t pad_mode;   /* MM_PAD_CONSTANT or MM_PAD_REFLECT */
    int32_t n_mels;
    int32_t n_mfcc;
    float f_min;
    float f_max;        /* <= 0: sr/2 */
    float top_db;       /* <= 0: no floor; mm_mfcc uses 80 */
    int32_t dft_form;   /* MM_DFT_FFT_F32 (0), MM_DFT_GEMM_BF16X3, MM_DFT_GEMM_BF16 or MM_DFT_GEMM_F16X3 */
} MMFrontEndParams;

/* MFCC of n_clips clips of any lengths in one batched launch sequence.
 * outs[i] receives [min(n_mfcc,n_mels), n_frames_i]; free each with
 * mm_buffer_free. */
MM_API int32_t mm_mfcc_batch(mm_context ctx, const float* const* signals, const int64_t* lengths,
                      int32_t n_clips, const MMFrontEndParams* params, MMBuffer* outs);

/* A plan fixes the parameters and clip lengths of a batch, keeps its tables
 * and device buffers resident and captures its launches in a CUDA graph.
 * Clip i's samples go to mm_plan_device_input() + mm_plan_input_offset(i)
 * floats, its [rows, n_frames_i] result is at mm_plan_device_output() +
 * mm_plan_output_offset(i) floats.  Streams are passed as void* (a
 * cudaStream_t; NULL = the plan's own). */
typedef void* mm_plan;

MM_API mm_plan mm_plan_create(mm_context ctx, const MMFrontEndParams* params,
                       const int64_t* lengths, int32_t n_clips, int32_t* status);
/* A plan over clips with their own parameters (clip_params[i] for clip i):
 * clips are grouped by parameter set, each group is cut into branches of at
 * most max_clips_per_branch clips (0: one branch per group), and the graph
 * runs the branches concurrently (one persistent launch sequence each, the
 * autotuned variant of its n_fft).  With host I/O every branch copies its own
 * clips in and out, so copies of one branch overlap kernels of another. */
MM_API mm_plan mm_plan_create_groups(mm_context ctx, const MMFrontEndParams* clip_params,
                                     const int64_t* lengths, int32_t n_clips,
                                     int32_t max_clips_per_branch, int32_t* status);
MM_API int32_t mm_plan_branches(mm_plan plan);
/* Output rows of clip i (min(n_mfcc, n_mels) of its parameters). */
MM_API int32_t mm_plan_clip_rows(mm_plan plan, int32_t clip);
MM_API void mm_plan_destroy(mm_plan plan);
MM_API float* mm_plan_device_input(mm_plan plan);
MM_API float* mm_plan_device_output(mm_plan plan);
MM_API int64_t mm_plan_input_offset(mm_plan plan, int32_t clip);
MM_API int64_t mm_plan_output_offset(mm_plan plan, int32_t clip);
MM_API int64_t mm_plan_clip_frames(mm_plan plan, int32_t clip);
/* Output rows shared by every clip, or -1 when the groups differ. */
MM_API int32_t mm_plan_rows(mm_plan plan);
MM_API int64_t mm_plan_total_frames(mm_plan plan);
MM_API int32_t mm_plan_kernel_launches(mm_plan plan);
/* (Plans of one branch.)  The log-mel intermediate of the last execution, frame-major
 * [total_frames, n_mels] (clip i's frames start at the sum of the earlier
 * clips' frame counts), before the top_db floor; and clip i's maximum dB. */
MM_API float* mm_plan_device_mel_db(mm_plan plan);
MM_API int32_t mm_plan_clip_max_db(mm_plan plan, int32_t clip, float* max_db);
/* (Any plan.)  Device address of clip i's log-mel rows of the last execution,
 * frame-major [n_frames_i, n_mels of its group], before the top_db floor;
 * NULL for an invalid clip. */
MM_API const float* mm_plan_clip_mel_db(mm_plan plan, int32_t clip);
/* Replays the captured graph on `stream`. */
MM_API int32_t mm_plan_execute(mm_plan plan, void* stream);
/* (Plans of one branch.)  Same kernels launched directly, with CUDA events
 * recorded around each of the three stages into timing slot `slot` (0..63);
 * read them after the stream has synchronised with mm_plan_stage_ms. */
MM_API int32_t mm_plan_execute_timed(mm_plan plan, void* stream, int32_t slot);
MM_API int32_t mm_plan_stage_ms(mm_plan plan, int32_t slot, float* ms3);
/* Host buffers in and out: copies signals[i] into the device input, runs the
 * plan, copies every clip's result into outs[i] and synchronises. */
/* Synchronises `stream` (NULL: the plan's own) and reports whether a bounded
 * wait of a tensor-core kernel of the plan (DFT-as-GEMM forms, launch variant
 * 5) ran out since the last report: MM_ERR_INTERNAL, else MM_OK.
 * mm_plan_execute_host reports the same itself. */
MM_API int32_t mm_plan_status(mm_plan plan, void* stream);
MM_API int32_t mm_plan_execute_host(mm_plan plan, const float* const* signals, float* const* outs,
                             void* stream);

/* Autotuning of the frame kernel's launch variant, process-wide per n_fft:
 * variants 0-2 are the CTA-per-tile kernel with different frames per CTA and
 * register budgets; variant 3 (MFCC path, n_fft 256..2048) is the
 * warp-per-frame kernel (warp pair at 4096); variant 5 (MFCC path, n_fft 2048)
 * is the tensor-core kernel (both 32-point DFT stages as fp16x3 tcgen05
 * GEMMs).  mm_autotune times every variant that applies on n_clips synthetic
 * clips of clip_samples samples (reps launches each), writes each variant's
 * milliseconds to variant_ms[variant] (6 entries; 0 for variants not timed),
 * keeps the fastest and returns it in *best_variant.  Plans and calls made
 * afterwards use the tuned variant. */
MM_API int32_t mm_autotune(mm_context ctx, const MMFrontEndParams* params, int64_t clip_samples,
                           int32_t n_clips, int32_t reps, float* variant_ms, int32_t* best_variant);
MM_API int32_t mm_tune_set(int32_t n_fft, int32_t variant);
MM_API int32_t mm_tune_get(int32_t n_fft);

/* ---- Serving: continuous batching with device-memory admission --------- */

/* Returned by mm_server_poll / mm_server_wait while a request is not done. */
#define MM_PENDING 1

/* A server owns a scheduler thread and max_inflight CUDA streams.  Requests
 * (one clip + its MFCC parameters each) are queued by mm_server_submit; the
 * scheduler groups pending requests by parameter set into batches (oldest
 * first, up to max_batch_clips and the free part of device_budget_bytes) and
 * starts a batch whenever a stream is free, so requests that arrive while
 * others run are admitted as streams and memory free up, and batches of
 * different groups overlap on the device.  Tables stay resident per group.
 * Results are identical to mm_mfcc_batch on the same clip.  All calls are
 * thread-safe; no call may be in progress while mm_server_destroy runs. */
typedef void* mm_server;

typedef struct {
    int64_t device_budget_bytes; /* device memory of the batches in flight; <= 0: 40 GiB */
    int32_t max_batch_clips;     /* <= 0: 256 */
    int32_t max_inflight;        /* batches on the device at once; <= 0: 4 (at most 64) */
    int64_t host_pinned_bytes;   /* pinned host memory for queued samples and batch results; <= 0: 8 GiB
                                    (past it, samples wait in pageable copies and results go
                                    through the batch slot's staging) */
} MMServerConfig;

typedef struct {
    int64_t submitted, completed, failed, pending, inflight_batches, batches_launched;
    int64_t bytes_in_use, peak_bytes_in_use;
    double audio_seconds_completed;
    double latency_p50_ms, latency_p99_ms, latency_mean_ms, latency_max_ms; /* submit -> result */
    double scheduler_launch_ms, scheduler_finish_ms; /* host time spent starting / reaping batches */
} MMServerStats;

MM_API mm_server mm_server_create(const MMServerConfig* config, int32_t* status);
/* Finishes the batches in flight, drops requests that never started and
 * frees every undelivered result. */
MM_API void mm_server_destroy(mm_server server);
/* Copies the samples (into pinned host memory while the pool has room);
 * *request_id identifies the request.  A request with no
 * frame or no coefficient is rejected (MM_ERR_INVALID_INPUT); a request
 * whose batch alone exceeds the budget fails with MM_ERR_ALLOC_FAILED. */
MM_API int32_t mm_server_submit(mm_server server, const float* signal, int64_t length,
                                const MMFrontEndParams* params, int64_t* request_id);
/* As mm_server_submit without the copy: the server reads `signal` (length
 * samples) in place when the request's batch starts.  The caller keeps the
 * buffer alive and unchanged until the request's result has been taken
 * (mm_server_poll / mm_server_wait returned other than MM_PENDING) or the
 * server is destroyed.  From pinned host memory (cudaMallocHost /
 * cudaHostRegister) the upload runs at full PCIe speed with no host copy. */
MM_API int32_t mm_server_submit_borrowed(mm_server server, const float* signal, int64_t length,
                                         const MMFrontEndParams* params, int64_t* request_id);
/* n borrowed submits in one call (params: one struct per request).  On an
 * error the requests before the failing one stay queued, the failing one and
 * those after it get request_ids -1, and its status is returned. */
MM_API int32_t mm_server_submit_borrowed_many(mm_server server, const float* const* signals,
                                              const int64_t* lengths, int32_t n,
                                              const MMFrontEndParams* params, int64_t* request_ids);
/* MM_PENDING while running; otherwise moves the result ([rows, n_frames],
 * free with mm_buffer_free) into *out, or returns the request's error, and
 * forgets the request. */
MM_API int32_t mm_server_poll(mm_server server, int64_t request_id, MMBuffer* out);
/* As mm_server_poll, waiting up to timeout_ms (< 0: no limit). */
MM_API int32_t mm_server_wait(mm_server server, int64_t request_id, int32_t timeout_ms, MMBuffer* out);
MM_API int32_t mm_server_stats(mm_server server, MMServerStats* out);
MM_API int32_t mm_server_reset_stats(mm_server server);

/* MFCC of one clip that is already in device memory, allocating nothing.
 * No counterpart in the reference.  For callers that must not allocate
 * device memory while they run (code inside another framework's memory pool
 * or under a hard memory budget, real-time audio threads that may not block
 * in the allocator, plugin hosts that forbid cudaMalloc/cudaFree): they pass
 * the signal (d_signal, 4-byte aligned, signal_length samples) and the output
 * d_out (min(n_mfcc, n_mels) x n_frames floats, row-major, n_frames as in
 * mm_mfcc); all scratch comes from a 16 MiB array built into the library,
 * which every GPU that loads the library holds until exit.  Same parameters,
 * sentinels and results as mm_mfcc.  Returns MM_ERR_INVALID_INPUT when the
 * clip's log-mel scratch plus tables exceed that array (about 31 000 frames,
 * 12 minutes at 22050 Hz with hop 512, for n_fft 2048 and 128 mels).  Work
 * is enqueued on `stream` (NULL = the default stream); d_out is ready after
 * the stream synchronises.  The array keeps the tables of the last parameter
 * set used on the device: a call with a new parameter set builds them there
 * and waits on `stream` once (for the filterbank size), a call that repeats
 * the previous parameters enqueues three kernels and does not wait.  The
 * first call on each device looks up the array's device address, so make
 * that first call before any stream capture; calls after a device reset are
 * not supported.  Calls share the array: calls whose work overlaps on the
 * GPU race. */
MM_API int32_t mm_mfcc_noalloc(const float* d_signal, int64_t signal_length, int32_t sample_rate,
                               int32_t n_mfcc, int32_t n_fft, int32_t hop_length, int32_t win_length,
                               int32_t n_mels, float f_min, float f_max, int32_t center, float* d_out,
                               void* stream);

#ifdef __cplusplus
}
#endif

#endif /* METALMOM_H */
