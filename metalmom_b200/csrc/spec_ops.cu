// Operations on a spectrogram the caller already has (additive entry points):
//
//   mm_mel_project   the S= path of melspectrogram: the Slaney filterbank
//                    applied to a given [n_freqs, n_frames] spectrogram
//                    (python/metalmom/feature.py:50-57, `_mel_fb.py` @ S);
//   mm_dct_ortho     the S= path of mfcc: DCT-II ortho along the rows of a
//                    given [n_rows, n_frames] log-mel spectrogram, first n_out
//                    rows (feature.py:130-134, scipy dct(type 2, 'ortho'));
//   mm_power_to_db_device / mm_amplitude_to_db_device
//                    dB scaling of a device buffer on the caller's stream, the
//                    reference value given or taken as max(S) on the device
//                    (ref=np.max, feature.py:247-248; Scaling.swift:73-118).
//
// The projection and the DCT are one thread per (output row, frame) with the
// frames of a warp consecutive, so every read of S and every write is
// coalesced along the frame axis; the filterbank row or basis row is a
// warp-uniform broadcast.  A frame whose column of S holds a non-finite value
// gives NaN in every band, as the dense product does (0 * inf = NaN).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "runtime.h"

namespace mm {

namespace {

constexpr int kColThreads = 128;  // frames per CTA

// bad[t] = 1 when column t of S holds a non-finite value.
__global__ void column_bad_kernel(const float *S, int n_rows, long long T, int *bad) {
  const long long t = blockIdx.x * (long long)kColThreads + threadIdx.x;
  if (t >= T) return;
  int b = 0;
  for (int k = 0; k < n_rows; k++) b |= !isfinite(S[(long long)k * T + t]);
  bad[t] = b;
}

// out[m][t] = sum_k W[m][k] S[k][t] over the nonzero range of row m.
__global__ void mel_project_kernel(const float *S, long long T, const float *W, const int4 *info, int nfreq,
                                   const int *bad, float *out) {
  const long long t = blockIdx.x * (long long)kColThreads + threadIdx.x;
  const int m = blockIdx.y;
  if (t >= T) return;
  const int4 in = __ldg(info + m);  // {first bin, count, -, NaN-row flag}
  const float *w = W + (long long)m * nfreq + in.x;
  const float *s = S + (long long)in.x * T + t;
  float a0 = 0.0f, a1 = 0.0f;
  int q = 0;
  for (; q + 1 < in.y; q += 2) {
    a0 = fmaf(__ldg(w + q), s[(long long)q * T], a0);
    a1 = fmaf(__ldg(w + q + 1), s[(long long)(q + 1) * T], a1);
  }
  if (q < in.y) a0 = fmaf(__ldg(w + q), s[(long long)q * T], a0);
  float acc = a0 + a1;
  if (in.w || bad[t]) acc = __int_as_float(0x7fc00000);
  out[(long long)m * T + t] = acc;
}

// out[k][t] = sum_n B[k][n] S[n][t].
__global__ void dct_cols_kernel(const float *S, long long T, const float *B, int n_rows, float *out) {
  const long long t = blockIdx.x * (long long)kColThreads + threadIdx.x;
  const int k = blockIdx.y;
  if (t >= T) return;
  const float *b = B + (long long)k * n_rows;
  float a0 = 0.0f, a1 = 0.0f;
  int n = 0;
  for (; n + 1 < n_rows; n += 2) {
    a0 = fmaf(__ldg(b + n), S[(long long)n * T + t], a0);
    a1 = fmaf(__ldg(b + n + 1), S[(long long)(n + 1) * T + t], a1);
  }
  if (n < n_rows) a0 = fmaf(__ldg(b + n), S[(long long)n * T + t], a0);
  out[(long long)k * T + t] = a0 + a1;
}

// Resident dense filterbanks for the projection, per (device, sr, n_fft,
// n_mels, fmin, fmax).
struct MelKey {
  int dev, sr, n_fft, n_mels;
  float fmin, fmax;
  bool operator<(const MelKey &o) const {
    return std::tie(dev, sr, n_fft, n_mels, fmin, fmax) < std::tie(o.dev, o.sr, o.n_fft, o.n_mels, o.fmin, o.fmax);
  }
};
struct MelDense {
  float *W = nullptr;
  int4 *info = nullptr;
};
std::mutex g_mel_mu;
std::map<MelKey, MelDense> g_mel;

int mel_dense(int sr, int n_fft, int n_mels, float fmin, float fmax, MelDense *out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  const MelKey key{dev, sr, n_fft, n_mels, fmin, fmax};
  std::lock_guard<std::mutex> lock(g_mel_mu);
  auto it = g_mel.find(key);
  if (it != g_mel.end()) {
    *out = it->second;
    return MM_OK;
  }
  MelDense d;
  const size_t nfreq = (size_t)(n_fft / 2 + 1);
  cudaStream_t s = nullptr;
  e = cudaMalloc(&d.W, sizeof(float) * nfreq * (size_t)n_mels);
  if (e == cudaSuccess) e = cudaMalloc(&d.info, sizeof(int4) * (size_t)n_mels);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = build_mel_dense(d.W, d.info, sr, n_fft, n_mels, fmin, fmax, s);
  if (s) {
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e2;
    cudaStreamDestroy(s);
  }
  if (e != cudaSuccess) {
    cudaFree(d.W);
    cudaFree(d.info);
    cudaGetLastError();
    return cuda_status(e);
  }
  g_mel[key] = d;
  *out = d;
  return MM_OK;
}

inline size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

// Host [n_rows, T] in, kernel(s) on the thread's stream, host [rows_out, T]
// out (malloc'd, owned by the MMBuffer).
template <typename Launch>
int32_t run_columns(const float *S, int n_rows, long long T, int rows_out, size_t extra_dev, Launch launch,
                    MMBuffer *out) {
  int st = gpu_available();
  if (st != MM_OK) return st;
  const size_t in_b = sizeof(float) * (size_t)n_rows * (size_t)T;
  const size_t out_b = sizeof(float) * (size_t)rows_out * (size_t)T;
  Workspace *ws = nullptr;
  if ((st = thread_workspace(up256(in_b) + up256(out_b) + up256(extra_dev), std::max(in_b, out_b), &ws)) != MM_OK)
    return st;
  cudaStream_t s = ws->stream;
  float *d_in = reinterpret_cast<float *>(ws->dev);
  float *d_out = reinterpret_cast<float *>(ws->dev + up256(in_b));
  char *d_extra = ws->dev + up256(in_b) + up256(out_b);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    memcpy(ws->host, S, in_b);
    e = cudaMemcpyAsync(d_in, ws->host, in_b, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = launch(d_in, d_out, d_extra, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ws->host, d_out, out_b, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return cuda_status(e);
  }
  float *res = (float *)malloc(out_b > 0 ? out_b : 1);
  if (!res) return MM_ERR_ALLOC_FAILED;
  memcpy(res, ws->host, out_b);
  fill_buffer(out, res, rows_out, T);
  return MM_OK;
}

int32_t db_device(const float *x, int64_t count, float mult, float ref, int32_t ref_mode, float amin, float top_db,
                  float *y, void *stream) {
  if (!x || !y || count <= 0 || (ref_mode != 0 && ref_mode != 1)) return MM_ERR_INVALID_INPUT;
  int st = gpu_available();
  if (st != MM_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned *slots = nullptr;  // {clip max, ref max, ref NaN flag}
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&slots), 4 * sizeof(unsigned), s);
  if (e != cudaSuccess) return cuda_status(e);
  e = launch_db(x, y, count, mult, amin, ref, top_db, slots, s, ref_mode ? slots + 1 : nullptr);
  const cudaError_t e2 = cudaFreeAsync(slots, s);
  if (e == cudaSuccess) e = e2;
  return e == cudaSuccess ? MM_OK : cuda_status(e);
}

}  // namespace

}  // namespace mm

using namespace mm;

extern "C" {

// melspectrogram(S=...) on the GPU (feature.py:50-57 of the reference builds the
// same Slaney filterbank in Python and multiplies).  S: [n_freqs, n_frames]
// row-major with n_freqs == n_fft / 2 + 1 (the reference's matmul fails
// otherwise); f_max <= 0 -> sr / 2.  Output [n_mels, n_frames]; n_mels == 0
// gives an empty [0, n_frames] result.
int32_t mm_mel_project(mm_context ctx, const float *S, int64_t count, int32_t n_freqs, int32_t n_frames,
                       int32_t sample_rate, int32_t n_fft, int32_t n_mels, float f_min, float f_max,
                       MMBuffer *out) {
  if (!ctx || !S || !out || n_freqs < 1 || n_frames < 1 || n_fft < 1 || n_mels < 0 || sample_rate <= 0)
    return MM_ERR_INVALID_INPUT;
  if (n_freqs != n_fft / 2 + 1 || count < (int64_t)n_freqs * n_frames) return MM_ERR_INVALID_INPUT;
  if (n_mels == 0) {
    fill_buffer(out, nullptr, 0, n_frames);
    return MM_OK;
  }
  int st = gpu_available();
  if (st != MM_OK) return st;
  const float fmax = f_max > 0.0f ? f_max : 0.5f * (float)sample_rate;
  MelDense d;
  if ((st = mel_dense(sample_rate, n_fft, n_mels, f_min, fmax, &d)) != MM_OK) return st;
  const long long T = n_frames;
  auto launch = [&](const float *d_in, float *d_out, char *d_extra, cudaStream_t s) {
    int *bad = reinterpret_cast<int *>(d_extra);
    const unsigned gx = (unsigned)((T + kColThreads - 1) / kColThreads);
    column_bad_kernel<<<gx, kColThreads, 0, s>>>(d_in, n_freqs, T, bad);
    mel_project_kernel<<<dim3(gx, (unsigned)n_mels), kColThreads, 0, s>>>(d_in, T, d.W, d.info, n_freqs, bad,
                                                                           d_out);
    return cudaGetLastError();
  };
  return run_columns(S, n_freqs, T, n_mels, sizeof(int) * (size_t)T, launch, out);
}

// mfcc(S=...) on the GPU (feature.py:130-134 of the reference: scipy
// dct(S, axis=0, type=2, norm='ortho')[:n_mfcc]).  S: [n_rows, n_frames];
// output [min(n_out, n_rows), n_frames].  No top_db floor (S is already in dB).
int32_t mm_dct_ortho(mm_context ctx, const float *S, int64_t count, int32_t n_rows, int32_t n_frames,
                     int32_t n_out, MMBuffer *out) {
  if (!ctx || !S || !out || n_rows < 1 || n_frames < 1 || n_out < 0) return MM_ERR_INVALID_INPUT;
  if (count < (int64_t)n_rows * n_frames) return MM_ERR_INVALID_INPUT;
  const int rows_out = std::min(n_out, n_rows);
  if (rows_out == 0) {
    fill_buffer(out, nullptr, 0, n_frames);
    return MM_OK;
  }
  const long long T = n_frames;
  auto launch = [&](const float *d_in, float *d_out, char *d_extra, cudaStream_t s) {
    float *B = reinterpret_cast<float *>(d_extra);
    cudaError_t e = build_dct_basis_rows(B, rows_out, n_rows, s);
    if (e != cudaSuccess) return e;
    const unsigned gx = (unsigned)((T + kColThreads - 1) / kColThreads);
    dct_cols_kernel<<<dim3(gx, (unsigned)rows_out), kColThreads, 0, s>>>(d_in, T, B, n_rows, d_out);
    return cudaGetLastError();
  };
  return run_columns(S, n_rows, T, rows_out, sizeof(float) * (size_t)rows_out * n_rows, launch, out);
}

// power_to_db of a device buffer on the caller's stream (asynchronous: the
// result is ready when the stream reaches it).  ref_mode 0: divide by `ref`;
// 1: by max(d_in), computed on the device (ref=np.max; NaN when d_in holds
// one).  top_db <= 0: no floor.  d_out may equal d_in.
int32_t mm_power_to_db_device(const float *d_in, int64_t count, float ref, int32_t ref_mode, float amin,
                              float top_db, float *d_out, void *stream) {
  return db_device(d_in, count, 10.0f, ref, ref_mode, amin, top_db, d_out, stream);
}

// amplitude_to_db of a device buffer (20 log10), as mm_power_to_db_device.
int32_t mm_amplitude_to_db_device(const float *d_in, int64_t count, float ref, int32_t ref_mode, float amin,
                                  float top_db, float *d_out, void *stream) {
  return db_device(d_in, count, 20.0f, ref, ref_mode, amin, top_db, d_out, stream);
}

}  // extern "C"
