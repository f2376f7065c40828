// extern "C" entry points of libmetalmom.so (declared in include/metalmom.h).
//
// The reference entry points keep MetalMom's validation order, sentinels,
// status codes, output shapes and ownership rules (Bridge.swift:16-492,
// 3695-3711); the work itself runs on the CUDA device.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <unordered_set>
#include <vector>

#include "runtime.h"

using namespace mm;

namespace {

// Context registry: makes mm_destroy idempotent (Bridge.swift:16-40).
struct Context {
  int magic = 0x4d4d4232;
};
std::mutex g_ctx_mu;
std::unordered_set<void *> g_ctx;

// Run one clip (n = 1) or a batch of clips through `g`; on success *outs[i]
// holds a malloc'd [rows x n_frames_i] block (NULL when empty).
int run_batch(const Group &g_in, const float *const *signals, const int64_t *lengths, int n,
              float **outs) {
  for (int i = 0; i < n; i++) outs[i] = nullptr;
  Group g = g_in;
  g.variant = group_variant(g);
  Layout L;
  make_layout(g, lengths, n, L);
  if (L.total_frames == 0 || L.out_elems == 0) return MM_OK;
  int st = gpu_available();
  if (st != MM_OK) return st;
  const DevTables *t = get_tables(g, &st);
  if (!t) return st;
  const size_t dev_bytes = arena_bytes(g, L);
  DevBatch probe;
  const size_t desc_bytes = carve_arena(g, L, nullptr, probe);
  const size_t sig_bytes = sizeof(float) * (size_t)L.sig_elems;
  const size_t out_bytes = sizeof(float) * (size_t)L.out_elems;
  const size_t host_bytes = std::max(sig_bytes + desc_bytes, out_bytes) + 256;
  Workspace *ws = nullptr;
  if ((st = thread_workspace(dev_bytes, host_bytes, &ws)) != MM_OK) return st;
  DevBatch b;
  carve_arena(g, L, ws->dev, b);
  cudaStream_t s = ws->stream;
  cudaError_t e = cudaStreamSynchronize(s);  // staging buffer is free again
  if (e != cudaSuccess) return cuda_status(e);
  // Signals: a large clip goes straight from the caller's (pageable) buffer,
  // where the driver overlaps its own staging with the transfer (measured
  // ~150 us for 2.6 MB, against ~210 us for a copy into pinned staging then
  // an upload); small clips are gathered in pinned memory and uploaded in
  // one copy.  Descriptors always come from pinned memory.
  // The staged region (which spans the large clips' slots too) is uploaded
  // first, so that the direct copies, later in stream order, land on top.
  char *h = ws->host;
  constexpr size_t kDirect = size_t(1) << 20;
  bool staged = false;
  for (int i = 0; i < n; i++) {
    const size_t bytes = sizeof(float) * (size_t)lengths[i];
    if (bytes < kDirect) {
      memcpy(h + sizeof(float) * (size_t)L.clips[i].sig_off, signals[i], bytes);
      staged = true;
    }
  }
  pack_descriptors(L, h + sig_bytes);
  if (staged && (e = cudaMemcpyAsync(b.signal, h, sig_bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_status(e);
  for (int i = 0; i < n; i++) {
    const size_t bytes = sizeof(float) * (size_t)lengths[i];
    if (bytes >= kDirect &&
        (e = cudaMemcpyAsync(b.signal + L.clips[i].sig_off, signals[i], bytes, cudaMemcpyHostToDevice, s)) !=
            cudaSuccess)
      return cuda_status(e);
  }
  if ((e = cudaMemcpyAsync(b.clips, h + sig_bytes, desc_bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_status(e);
  if ((e = enqueue_batch(g, L, t, b, s, nullptr, nullptr)) != cudaSuccess) return cuda_status(e);
  if ((e = cudaMemcpyAsync(h, b.out, out_bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_status(e);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_status(e);
  if ((st = take_error_word(g, t)) != MM_OK) return st;  // a bounded wait of a tensor-core kernel ran out
  const int rows = output_rows(g);
  for (int i = 0; i < n; i++) {
    const size_t cnt = (size_t)rows * (size_t)L.clips[i].n_frames;
    if (cnt == 0) continue;
    outs[i] = (float *)malloc(sizeof(float) * cnt);
    if (!outs[i]) {
      for (int q = 0; q < i; q++) free(outs[q]), outs[q] = nullptr;
      return MM_ERR_ALLOC_FAILED;
    }
    memcpy(outs[i], h + sizeof(float) * (size_t)L.clips[i].out_off, sizeof(float) * cnt);
  }
  return MM_OK;
}

// Resolve the mel / MFCC sentinels (Bridge.swift:340-345, 432-437).
int resolve_mel_group(Group &g, int sr, int n_fft, int hop, int win, int center, int n_mels,
                      float fmin, float fmax) {
  if (n_fft <= 0 || n_mels < 0) return MM_ERR_INVALID_INPUT;
  g.sr = sr;
  g.n_fft = n_fft;
  g.log2n = ilog2(n_fft);
  g.hop = hop > 0 ? hop : n_fft / 4;
  g.win = win > 0 ? win : n_fft;
  g.window_zero = 0;
  g.center = center != 0;
  g.pad_mode = PAD_CONSTANT;
  g.n_mels = n_mels;
  g.fmin = fmin;
  g.fmax = fmax > 0.0f ? fmax : (float)sr / 2.0f;
  if (g.hop <= 0) return MM_ERR_INVALID_INPUT;  // the reference divides by zero here
  return MM_OK;
}

bool supported_size(const Group &g) { return g.log2n <= 15; }

}  // namespace

extern "C" {

mm_context mm_init(void) {
  Context *c = new (std::nothrow) Context();
  if (!c) return nullptr;
  std::lock_guard<std::mutex> lock(g_ctx_mu);
  g_ctx.insert(c);
  return c;
}

void mm_destroy(mm_context ctx) {
  if (!ctx) return;
  {
    std::lock_guard<std::mutex> lock(g_ctx_mu);
    if (g_ctx.erase(ctx) == 0) return;  // already destroyed
  }
  delete static_cast<Context *>(ctx);
}

void mm_buffer_free(MMBuffer *buf) {
  if (!buf) return;
  free(buf->data);
  buf->data = nullptr;
  buf->ndim = 0;
  buf->dtype = 0;
  buf->count = 0;
  for (int i = 0; i < 8; i++) buf->shape[i] = 0;
}

int32_t mm_stft(mm_context ctx, const float *signal_data, int64_t signal_length, int32_t sample_rate,
                const MMSTFTParams *params, MMBuffer *out) {
  if (!ctx || !signal_data || signal_length <= 0 || !params || !out) return MM_ERR_INVALID_INPUT;
  const int n_fft = params->n_fft;
  if (!is_pow2(n_fft)) return MM_ERR_INVALID_INPUT;
  Group g;
  g.mode = MODE_SPECTRUM;
  g.power = 1.0f;
  g.sr = sample_rate;
  g.n_fft = n_fft;
  g.log2n = ilog2(n_fft);
  g.hop = params->hop_length;
  g.win = params->win_length;
  g.window_zero = params->win_length <= 0;
  g.center = params->center != 0;
  g.n_mels = 0;
  g.n_mfcc_eff = 0;
  if (g.hop <= 0 || !supported_size(g)) return MM_ERR_INVALID_INPUT;
  const long long T = frame_count(signal_length, n_fft, g.hop, g.center);
  const long long rows = n_fft / 2 + 1;
  float *data = nullptr;
  if (T > 0) {
    int st = run_batch(g, &signal_data, &signal_length, 1, &data);
    if (st != MM_OK) return st;
  }
  fill_buffer(out, data, rows, T);
  return MM_OK;
}

// Complex STFT (additive; the C-ABI form of STFT.computeComplex,
// Spectral/STFT.swift:512-668): zero centre padding, the analysis window of
// mm_stft, X[k] = sum_n x[n] w[n] e^{-2 pi i k n / n_fft} with the imaginary
// parts of DC and Nyquist set to 0.  out: float32 [n_freqs][n_frames][2]
// (interleaved re, im: the layout mm_istft takes), ndim 3.  hop_length <= 0
// and win_length <= 0 take computeComplex's defaults (n_fft / 4, n_fft).  A
// non-power-of-two n_fft, or a signal shorter than one frame, gives MM_OK with
// shape [n_freqs, 0, 2], as computeComplex returns an empty [n_freqs, 0] signal.
int32_t mm_stft_complex(mm_context ctx, const float *signal_data, int64_t signal_length, int32_t sample_rate,
                        const MMSTFTParams *params, MMBuffer *out) {
  if (!ctx || !signal_data || signal_length <= 0 || !params || !out) return MM_ERR_INVALID_INPUT;
  const int n_fft = params->n_fft;
  if (n_fft <= 0) return MM_ERR_INVALID_INPUT;
  const long long nfreq = n_fft / 2 + 1;
  Group g;
  g.mode = MODE_COMPLEX;
  g.power = 1.0f;
  g.sr = sample_rate;
  g.n_fft = n_fft;
  g.log2n = is_pow2(n_fft) ? ilog2(n_fft) : 0;
  g.hop = params->hop_length > 0 ? params->hop_length : n_fft / 4;
  g.win = params->win_length > 0 ? params->win_length : n_fft;
  g.window_zero = 0;
  g.center = params->center != 0;
  g.n_mels = 0;
  g.n_mfcc_eff = 0;
  if (g.hop <= 0) return MM_ERR_INVALID_INPUT;
  const long long T = is_pow2(n_fft) ? frame_count(signal_length, n_fft, g.hop, g.center) : 0;
  if (T > 0 && !supported_size(g)) return MM_ERR_INVALID_INPUT;
  float *data = nullptr;
  if (T > 0) {
    int st = run_batch(g, &signal_data, &signal_length, 1, &data);
    if (st != MM_OK) return st;
  }
  fill_buffer(out, data, nfreq, T);
  out->ndim = 3;
  out->shape[2] = 2;
  out->count = 2 * nfreq * T;
  return MM_OK;
}

static int32_t db_common(const float *data, int64_t count, float mult, float ref, float amin,
                         float top_db, MMBuffer *out) {
  if (!data || count <= 0 || !out) return MM_ERR_INVALID_INPUT;
  int st = gpu_available();
  if (st != MM_OK) return st;
  const size_t bytes = sizeof(float) * (size_t)count;
  const size_t seg = ((bytes + 255) / 256) * 256;
  Workspace *ws = nullptr;
  if ((st = thread_workspace(2 * seg + 256, bytes, &ws)) != MM_OK) return st;
  cudaStream_t s = ws->stream;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e);
  float *d_x = reinterpret_cast<float *>(ws->dev);
  float *d_y = reinterpret_cast<float *>(ws->dev + seg);
  unsigned *slot = reinterpret_cast<unsigned *>(ws->dev + 2 * seg);
  memcpy(ws->host, data, bytes);
  if ((e = cudaMemcpyAsync(d_x, ws->host, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cuda_status(e);
  if ((e = launch_db(d_x, d_y, count, mult, amin, ref, top_db, slot, s)) != cudaSuccess)
    return cuda_status(e);
  if ((e = cudaMemcpyAsync(ws->host, d_y, bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_status(e);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_status(e);
  float *res = (float *)malloc(bytes);
  if (!res) return MM_ERR_ALLOC_FAILED;
  memcpy(res, ws->host, bytes);
  fill_buffer(out, res, count, 0);
  out->ndim = 1;
  out->shape[1] = 0;
  out->count = count;
  return MM_OK;
}

int32_t mm_power_to_db(mm_context ctx, const float *data, int64_t count, float ref, float amin,
                       float top_db, MMBuffer *out) {
  (void)ctx;  // the reference does not check the context here (Bridge.swift:276-278)
  return db_common(data, count, 10.0f, ref, amin, top_db, out);
}

int32_t mm_amplitude_to_db(mm_context ctx, const float *data, int64_t count, float ref, float amin,
                           float top_db, MMBuffer *out) {
  (void)ctx;
  return db_common(data, count, 20.0f, ref, amin, top_db, out);
}

int32_t mm_mel_spectrogram(mm_context ctx, const float *signal_data, int64_t signal_length,
                           int32_t sample_rate, int32_t n_fft, int32_t hop_length, int32_t win_length,
                           int32_t center, float power, int32_t n_mels, float f_min, float f_max,
                           MMBuffer *out) {
  if (!ctx || !signal_data || signal_length <= 0 || !out) return MM_ERR_INVALID_INPUT;
  Group g;
  int st = resolve_mel_group(g, sample_rate, n_fft, hop_length, win_length, center, n_mels, f_min, f_max);
  if (st != MM_OK) return st;
  g.mode = MODE_MEL;
  g.power = power;
  g.n_mfcc_eff = 0;
  const long long T = frame_count(signal_length, g.n_fft, g.hop, g.center);
  float *data = nullptr;
  if (T > 0 && n_mels > 0) {
    if (!supported_size(g)) return MM_ERR_INVALID_INPUT;
    st = run_batch(g, &signal_data, &signal_length, 1, &data);
    if (st != MM_OK) return st;
  }
  fill_buffer(out, data, n_mels, T);
  return MM_OK;
}

int32_t mm_mfcc(mm_context ctx, const float *signal_data, int64_t signal_length, int32_t sample_rate,
                int32_t n_mfcc, int32_t n_fft, int32_t hop_length, int32_t win_length, int32_t n_mels,
                float f_min, float f_max, int32_t center, MMBuffer *out) {
  if (!ctx || !signal_data || signal_length <= 0 || !out) return MM_ERR_INVALID_INPUT;
  Group g;
  int st = resolve_mel_group(g, sample_rate, n_fft, hop_length, win_length, center, n_mels, f_min, f_max);
  if (st != MM_OK) return st;
  if (n_mfcc < 0) return MM_ERR_INVALID_INPUT;
  g.mode = MODE_MELDB;
  g.power = 2.0f;
  g.amin = 1e-10f;
  g.ref = 1.0f;
  g.top_db = 80.0f;
  g.n_mfcc_eff = std::min(n_mfcc, n_mels);
  const long long T = frame_count(signal_length, g.n_fft, g.hop, g.center);
  float *data = nullptr;
  if (T > 0 && g.n_mfcc_eff > 0) {
    if (!supported_size(g)) return MM_ERR_INVALID_INPUT;
    st = run_batch(g, &signal_data, &signal_length, 1, &data);
    if (st != MM_OK) return st;
  }
  fill_buffer(out, data, g.n_mfcc_eff, T);
  return MM_OK;
}

}  // extern "C"

// Savitzky-Golay derivative coefficients in float64 (Delta.swift:30-135):
// row `order` of (V^T V)^-1 V^T with V[i][j] = (i - width/2)^j, j <= order,
// times order!.  False when V^T V is singular.
static bool savgol_coeffs(int width, int order, float *out) {
  const int cols = order + 1, half = width / 2;
  std::vector<double> V((size_t)width * cols), A((size_t)cols * 2 * cols, 0.0);
  for (int i = 0; i < width; i++) {
    double p = 1.0;
    for (int j = 0; j < cols; j++, p *= (double)(i - half)) V[(size_t)i * cols + j] = p;
  }
  for (int i = 0; i < cols; i++) {
    for (int j = 0; j < cols; j++) {
      double s = 0.0;
      for (int k = 0; k < width; k++) s += V[(size_t)k * cols + i] * V[(size_t)k * cols + j];
      A[(size_t)i * 2 * cols + j] = s;
    }
    A[(size_t)i * 2 * cols + cols + i] = 1.0;
  }
  for (int i = 0; i < cols; i++) {  // Gauss-Jordan with partial pivoting
    int piv = i;
    for (int k = i + 1; k < cols; k++)
      if (fabs(A[(size_t)k * 2 * cols + i]) > fabs(A[(size_t)piv * 2 * cols + i])) piv = k;
    if (piv != i)
      for (int j = 0; j < 2 * cols; j++) std::swap(A[(size_t)i * 2 * cols + j], A[(size_t)piv * 2 * cols + j]);
    const double d = A[(size_t)i * 2 * cols + i];
    if (fabs(d) <= 1e-15) return false;
    for (int j = 0; j < 2 * cols; j++) A[(size_t)i * 2 * cols + j] /= d;
    for (int k = 0; k < cols; k++) {
      if (k == i) continue;
      const double f = A[(size_t)k * 2 * cols + i];
      for (int j = 0; j < 2 * cols; j++) A[(size_t)k * 2 * cols + j] -= f * A[(size_t)i * 2 * cols + j];
    }
  }
  double fact = 1.0;
  for (int i = 2; i <= order; i++) fact *= (double)i;
  for (int k = 0; k < width; k++) {
    double s = 0.0;
    for (int j = 0; j < cols; j++) s += A[(size_t)order * 2 * cols + cols + j] * V[(size_t)k * cols + j];
    out[k] = (float)(s * fact);
  }
  return true;
}

// Host matrix in -> kernel -> host matrix out through the thread's workspace.
template <typename Launch>
static int32_t run_matrix(const float *data, size_t in_count, size_t out_count, long long rows, long long cols,
                          MMBuffer *out, Launch launch) {
  int st = gpu_available();
  if (st != MM_OK) return st;
  const size_t in_b = sizeof(float) * in_count, out_b = sizeof(float) * out_count;
  const size_t in_pad = (in_b + 255) & ~size_t(255);
  Workspace *ws = nullptr;
  if ((st = thread_workspace(in_pad + out_b, std::max(in_b, out_b), &ws)) != MM_OK) return st;
  cudaStream_t s = ws->stream;
  cudaError_t e = cudaStreamSynchronize(s);
  float *d_in = reinterpret_cast<float *>(ws->dev), *d_out = reinterpret_cast<float *>(ws->dev + in_pad);
  if (e == cudaSuccess) {
    memcpy(ws->host, data, in_b);
    e = cudaMemcpyAsync(d_in, ws->host, in_b, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = launch(d_in, d_out, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ws->host, d_out, out_b, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e);
  float *res = (float *)malloc(out_b);
  if (!res) return MM_ERR_ALLOC_FAILED;
  memcpy(res, ws->host, out_b);
  fill_buffer(out, res, rows, cols);
  return MM_OK;
}

extern "C" {

// ---------------------------------------------------------------------------
// features on the front end: onset strength, delta, stack_memory
// ---------------------------------------------------------------------------

// Replaces Bridge.swift:1319-1358 (mm_onset_strength).  Sentinels as there:
// hop <= 0 -> 512, f_max <= 0 -> sr/2; window n_fft, lag 1, power_to_db with
// ref 1, amin 1e-10, top_db 80.  Shape [1, n_frames] (aggregate) or
// [n_mels, n_frames]; [1, 1] / [n_mels, 1] zeros when there are no frames.
int32_t mm_onset_strength(mm_context ctx, const float *signal_data, int64_t signal_length, int32_t sample_rate,
                          int32_t n_fft, int32_t hop_length, int32_t n_mels, float f_min, float f_max,
                          int32_t center, int32_t aggregate, MMBuffer *out) {
  (void)ctx;  // the reference ignores the context here too
  if (!signal_data || signal_length <= 0 || !out) return MM_ERR_INVALID_INPUT;
  if (n_mels <= 0) return MM_ERR_INVALID_INPUT;  // the reference would average over no bands
  Group g;
  int st = resolve_mel_group(g, sample_rate, n_fft, hop_length > 0 ? hop_length : 512, n_fft, center, n_mels,
                             f_min, f_max);
  if (st != MM_OK) return st;
  g.mode = MODE_MELDB;
  g.power = 2.0f;
  g.amin = 1e-10f;
  g.ref = 1.0f;
  g.top_db = 80.0f;
  g.post = aggregate ? POST_ONSET_MEAN : POST_ONSET_BANDS;
  g.lag = 1;
  g.n_mfcc_eff = 0;
  const int rows = aggregate ? 1 : n_mels;
  const long long T = frame_count(signal_length, g.n_fft, g.hop, g.center);
  float *data = nullptr;
  if (T > 0) {
    if (!supported_size(g)) return MM_ERR_INVALID_INPUT;
    st = run_batch(g, &signal_data, &signal_length, 1, &data);
    if (st != MM_OK) return st;
    fill_buffer(out, data, rows, T);
    return MM_OK;
  }
  data = (float *)calloc((size_t)rows, sizeof(float));
  if (!data) return MM_ERR_ALLOC_FAILED;
  fill_buffer(out, data, rows, 1);
  return MM_OK;
}

// Replaces Bridge.swift:934-955 (mm_delta): [n_features, n_frames] in and out.
// Rejected with MM_ERR_INVALID_INPUT where the reference traps: count !=
// n_features * n_frames, width even, < 3 or > 63, order < 1 or >= width,
// n_frames < width.
int32_t mm_delta(mm_context ctx, const float *data, int64_t count, int32_t n_features, int32_t n_frames,
                 int32_t width, int32_t order, MMBuffer *out) {
  (void)ctx;
  if (!data || count <= 0 || !out || n_features <= 0 || n_frames <= 0) return MM_ERR_INVALID_INPUT;
  if ((long long)n_features * n_frames != count) return MM_ERR_INVALID_INPUT;
  if (width < 3 || width % 2 == 0 || width > kDeltaMaxWidth || order < 1 || order >= width || n_frames < width)
    return MM_ERR_INVALID_INPUT;
  DeltaCoeffs c{};
  if (!savgol_coeffs(width, order, c.c)) return MM_ERR_INVALID_INPUT;
  return run_matrix(data, (size_t)count, (size_t)count, n_features, n_frames, out,
                    [&](const float *x, float *y, cudaStream_t s) {
                      return launch_delta(x, y, n_features, n_frames, width, c, s);
                    });
}

// Replaces Bridge.swift:959-980 (mm_stack_memory): [n_features * n_steps,
// n_frames], zeros before the start.
int32_t mm_stack_memory(mm_context ctx, const float *data, int64_t count, int32_t n_features, int32_t n_frames,
                        int32_t n_steps, int32_t delay, MMBuffer *out) {
  (void)ctx;
  if (!data || count <= 0 || !out || n_features <= 0 || n_frames <= 0 || n_steps <= 0) return MM_ERR_INVALID_INPUT;
  if ((long long)n_features * n_frames != count) return MM_ERR_INVALID_INPUT;
  const size_t out_count = (size_t)count * (size_t)n_steps;
  return run_matrix(data, (size_t)count, out_count, (long long)n_features * n_steps, n_frames, out,
                    [&](const float *x, float *y, cudaStream_t s) {
                      return launch_stack_memory(x, y, n_features, n_frames, n_steps, delay, s);
                    });
}

// ---------------------------------------------------------------------------
// additive: batches and plans
// ---------------------------------------------------------------------------
}  // extern "C"

int mm::resolve_frontend(const MMFrontEndParams *p, Group &g) {
  if (!p) return MM_ERR_INVALID_INPUT;
  int st = resolve_mel_group(g, p->sample_rate, p->n_fft, p->hop_length, p->win_length, p->center,
                             p->n_mels, p->f_min, p->f_max);
  if (st != MM_OK) return st;
  if (p->n_mfcc < 0 || (p->pad_mode != MM_PAD_CONSTANT && p->pad_mode != MM_PAD_REFLECT))
    return MM_ERR_INVALID_INPUT;
  if (!is_pow2(p->n_fft) || !supported_size(g)) return MM_ERR_INVALID_INPUT;
  if (p->dft_form < MM_DFT_FFT_F32 || p->dft_form > MM_DFT_GEMM_F16X3) return MM_ERR_INVALID_INPUT;
  if (p->dft_form != MM_DFT_FFT_F32 && !dft_supported(g.n_fft, g.win)) return MM_ERR_INVALID_INPUT;
  g.dft_form = p->dft_form;
  g.mode = MODE_MELDB;
  g.pad_mode = p->pad_mode;
  g.power = 2.0f;
  g.amin = 1e-10f;
  g.ref = 1.0f;
  g.top_db = p->top_db;
  g.n_mfcc_eff = std::min(p->n_mfcc, p->n_mels);
  return MM_OK;
}

extern "C" {

int32_t mm_mfcc_batch(mm_context ctx, const float *const *signals, const int64_t *lengths,
                      int32_t n_clips, const MMFrontEndParams *params, MMBuffer *outs) {
  if (!ctx || !signals || !lengths || n_clips <= 0 || !outs) return MM_ERR_INVALID_INPUT;
  for (int i = 0; i < n_clips; i++)
    if (!signals[i] || lengths[i] <= 0) return MM_ERR_INVALID_INPUT;
  Group g;
  int st = resolve_frontend(params, g);
  if (st != MM_OK) return st;
  std::vector<float *> data(n_clips, nullptr);
  if (g.n_mfcc_eff > 0) {
    st = run_batch(g, signals, lengths, n_clips, data.data());
    if (st != MM_OK) return st;
  }
  for (int i = 0; i < n_clips; i++)
    fill_buffer(&outs[i], data[i], g.n_mfcc_eff, frame_count(lengths[i], g.n_fft, g.hop, g.center));
  return MM_OK;
}

int32_t mm_tune_set(int32_t n_fft, int32_t variant) {
  if (!is_pow2(n_fft) || ilog2(n_fft) > 15 || variant < 0 ||
      (variant > kWarpVariant && !(variant == kTcVariant && n_fft == 2048)))
    return MM_ERR_INVALID_INPUT;
  set_tuned_variant(ilog2(n_fft), variant);
  return MM_OK;
}

int32_t mm_tune_get(int32_t n_fft) {
  if (!is_pow2(n_fft) || ilog2(n_fft) > 15) return MM_ERR_INVALID_INPUT;
  return tuned_variant(ilog2(n_fft));
}

int32_t mm_autotune(mm_context ctx, const MMFrontEndParams *params, int64_t clip_samples,
                    int32_t n_clips, int32_t reps, float *variant_ms, int32_t *best_variant) {
  if (!ctx || clip_samples <= 0 || n_clips <= 0 || reps <= 0) return MM_ERR_INVALID_INPUT;
  Group g;
  int st = resolve_frontend(params, g);
  if (st != MM_OK) return st;
  if ((st = gpu_available()) != MM_OK) return st;
  const DevTables *t = get_tables(g, &st);
  if (!t) return st;
  const int nv = frame_variants(g.log2n, g.mode, 1);
  // candidates: the frame variants, and the tensor-core kernel where it applies
  std::vector<int> cand;
  for (int v = 0; v < nv; v++) cand.push_back(v);
  if (g.log2n == 11 && g.mode == MODE_MELDB && g.dft_form == DFT_FFT_F32) cand.push_back(kTcVariant);
  std::vector<int64_t> lengths(n_clips, clip_samples);
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float best_ms = 0.0f;
  int best = 0;
  for (size_t ci = 0; ci < cand.size() && e == cudaSuccess; ci++) {
    const int v = cand[ci];
    Group gv = g;
    gv.variant = v;
    Layout L;
    make_layout(gv, lengths.data(), n_clips, L);
    char *arena = nullptr;
    e = cudaMalloc(&arena, arena_bytes(gv, L));
    if (e != cudaSuccess) break;
    DevBatch b;
    const size_t desc = carve_arena(gv, L, arena, b);
    std::vector<char> host(desc + 16);
    pack_descriptors(L, host.data());
    e = cudaMemcpyAsync(b.clips, host.data(), desc, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_fill_pattern(b.signal, L.sig_elems, s);
    for (int w = 0; w < 2 && e == cudaSuccess; w++) e = enqueue_batch(gv, L, t, b, s, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = enqueue_batch(gv, L, t, b, s, nullptr, nullptr);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaFree(arena);
    ms /= reps;
    if (variant_ms) variant_ms[v] = ms;
    if (e == cudaSuccess && (ci == 0 || ms < best_ms)) {
      best_ms = ms;
      best = v;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) return cuda_status(e);
  set_tuned_variant(g.log2n, best);
  if (best_variant) *best_variant = best;
  return MM_OK;
}

}  // extern "C"
