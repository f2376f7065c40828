// Inverse STFT on the GPU (mm_istft), the reverse direction of the front
// end: STFT.inverse (Spectral/STFT.swift:686-860) behind Bridge.swift:144-223.
//
// 1. istft_frames_kernel, one CTA per frame: the frame's bins X[0..M]
//    (M = n_fft/2, imaginary parts of DC and Nyquist dropped as the reference's
//    packed format does) become the M-point complex sequence
//    Z[k] = E[k] + i O[k], E = (X[k] + conj X[M-k]) / 2,
//    O = (X[k] - conj X[M-k]) e^{+2 pi i k / n_fft} / 2, whose inverse DFT z
//    gives the real frame x[2n] = Re z[n], x[2n+1] = Im z[n]; the inverse DFT
//    is an in-place radix-2 transform in shared memory; the frame times the
//    synthesis window is stored frame-major.
// 2. istft_ola_kernel, one thread per output sample: the overlapping frames'
//    samples and squared window values are summed in frame order, the sum is
//    divided by the window sum where that exceeds 1e-10, and the centre padding
//    / requested length are applied.  Gathering per output sample keeps the
//    result deterministic (no atomics).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "runtime.h"

namespace mm {

// T[t] = exp(+2 pi i t / n_fft) (float64, rounded once) and the synthesis
// window prepared as the analysis window (STFT.swift:44-57).
__global__ void istft_tables_kernel(float2 *tw, float *w, int n_fft, int win) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_fft) return;
  double s, c;
  sincospi(2.0 * (double)t / (double)n_fft, &s, &c);
  tw[t] = make_float2((float)c, (float)s);
  double v = 0.0;
  if (win > 0) {
    long long idx = t;
    if (win < n_fft) idx = (long long)t - (n_fft - win) / 2;
    else if (win > n_fft) idx = (long long)t + (win - n_fft) / 2;
    if (idx >= 0 && idx < win) v = (win == 1) ? 1.0 : 0.5 - 0.5 * cospi(2.0 * (double)idx / (double)win);
  }
  w[t] = (float)v;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__global__ void __launch_bounds__(256) istft_frames_kernel(const float2 *S, int n_frames, int n_fft,
                                                             int log2m, const float2 *tw, const float *w,
                                                             float *frames) {
  extern __shared__ float2 z[];  // M complex
  const int M = n_fft / 2;
  const int f = blockIdx.x;
  // bins of this frame: S[k * n_frames + f] (row-major [n_freqs][n_frames])
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    float2 a = S[(long long)k * n_frames + f];
    float2 b = S[(long long)(M - k) * n_frames + f];
    if (k == 0) {  // DC and Nyquist carry real parts only
      a.y = 0.0f;
      b.y = 0.0f;
    }
    const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
    const float2 d = make_float2(0.5f * (a.x - b.x), 0.5f * (a.y + b.y));  // (X[k] - conj X[M-k]) / 2
    const float2 o = cmulf(d, tw[k]);                                     // * e^{+2 pi i k / n_fft}
    const float2 zk = make_float2(e.x - o.y, e.y + o.x);                  // E + i O
    const unsigned r = log2m > 0 ? (__brev((unsigned)k) >> (32 - log2m)) : 0u;
    z[r] = zk;
  }
  __syncthreads();
  // in-place radix-2 inverse DFT (decimation in time, bit-reversed input)
  for (int len = 2; len <= M; len <<= 1) {
    const int half = len >> 1, stride = n_fft / len;  // W_len^-j = T[j * n_fft / len]
    for (int b = threadIdx.x; b < M / 2; b += blockDim.x) {
      const int grp = b / half, j = b - grp * half;
      const int i0 = grp * len + j, i1 = i0 + half;
      const float2 t = cmulf(z[i1], tw[j * stride]);
      const float2 u = z[i0];
      z[i0] = make_float2(u.x + t.x, u.y + t.y);
      z[i1] = make_float2(u.x - t.x, u.y - t.y);
    }
    __syncthreads();
  }
  const float inv = 1.0f / (float)M;
  float *dst = frames + (long long)f * n_fft;
  for (int n = threadIdx.x; n < M; n += blockDim.x) {
    const float2 v = z[n];
    dst[2 * n] = v.x * inv * w[2 * n];
    dst[2 * n + 1] = v.y * inv * w[2 * n + 1];
  }
}

__global__ void istft_ola_kernel(const float *frames, const float *w, int n_frames, int n_fft, int hop,
                                 long long expected, long long trim, long long out_len, float *out) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < out_len;
       s += (long long)gridDim.x * blockDim.x) {
    const long long p = s + trim;
    float v = 0.0f;
    if (p < expected) {
      const long long f_lo = p - n_fft + 1 <= 0 ? 0 : (p - n_fft + 1 + hop - 1) / hop;
      const long long last = p / hop;
      const long long f_hi = last < n_frames - 1 ? last : (long long)n_frames - 1;
      float acc = 0.0f, ws = 0.0f;
      for (long long f = f_lo; f <= f_hi; f++) {
        const int j = (int)(p - f * hop);
        acc += frames[f * n_fft + j];
        const float wj = w[j];
        ws += wj * wj;
      }
      v = ws > 1e-10f ? acc / ws : acc;
    }
    out[s] = v;
  }
}

}  // namespace mm

using namespace mm;

extern "C" {

// Replaces Bridge.swift:144-223 (mm_istft).  stft_data: interleaved complex
// [n_freqs, n_frames] row-major (2 * n_freqs * n_frames floats).  Output ndim 1.
// Rejected with MM_ERR_INVALID_INPUT where the reference would misbehave:
// n_freqs < 2, n_frames < 1, stft_count < 2 * n_freqs * n_frames, hop <= 0,
// n_fft > 32768.  A non-power-of-two n_fft gives zeros, as in the reference.
int32_t mm_istft(mm_context ctx, const float *stft_data, int64_t stft_count, int32_t n_freqs, int32_t n_frames,
                 int32_t sample_rate, int32_t hop_length, int32_t win_length, int32_t center, int64_t output_length,
                 MMBuffer *out) {
  (void)sample_rate;
  if (!ctx || !stft_data || stft_count <= 0 || !out) return MM_ERR_INVALID_INPUT;
  if (n_freqs < 2 || n_frames < 1 || hop_length <= 0) return MM_ERR_INVALID_INPUT;
  if (stft_count < 2LL * n_freqs * n_frames) return MM_ERR_INVALID_INPUT;
  const int n_fft = (n_freqs - 1) * 2;
  if (n_fft > 32768) return MM_ERR_INVALID_INPUT;
  const long long expected = (long long)n_fft + (long long)(n_frames - 1) * hop_length;
  long long trim = 0, out_len = 0;
  if (center) {
    trim = n_fft / 2;
    out_len = output_length > 0 ? output_length : std::max<long long>(0, expected - n_fft);
  } else {
    out_len = output_length > 0 ? output_length : expected;
  }
  for (int i = 0; i < 8; i++) out->shape[i] = 0;
  out->ndim = 1;
  out->dtype = 0;
  if (out_len <= 0) {
    out->data = nullptr;
    out->count = 0;
    return MM_OK;
  }
  float *res = (float *)calloc((size_t)out_len, sizeof(float));
  if (!res) return MM_ERR_ALLOC_FAILED;
  if (is_pow2(n_fft)) {
    int st = gpu_available();
    if (st != MM_OK) {
      free(res);
      return st;
    }
    const size_t in_b = sizeof(float) * 2 * (size_t)n_freqs * n_frames;
    const size_t tw_b = sizeof(float2) * (size_t)n_fft, w_b = sizeof(float) * (size_t)n_fft;
    const size_t fr_b = sizeof(float) * (size_t)n_fft * n_frames, out_b = sizeof(float) * (size_t)out_len;
    auto up = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t dev_b = up(in_b) + up(tw_b) + up(w_b) + up(fr_b) + up(out_b);
    Workspace *ws = nullptr;
    if ((st = thread_workspace(dev_b, std::max(in_b, out_b), &ws)) != MM_OK) {
      free(res);
      return st;
    }
    cudaStream_t s = ws->stream;
    char *p = ws->dev;
    float2 *d_S = reinterpret_cast<float2 *>(p);
    p += up(in_b);
    float2 *d_tw = reinterpret_cast<float2 *>(p);
    p += up(tw_b);
    float *d_w = reinterpret_cast<float *>(p);
    p += up(w_b);
    float *d_fr = reinterpret_cast<float *>(p);
    p += up(fr_b);
    float *d_out = reinterpret_cast<float *>(p);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) {
      memcpy(ws->host, stft_data, in_b);
      e = cudaMemcpyAsync(d_S, ws->host, in_b, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) {
      istft_tables_kernel<<<(n_fft + 255) / 256, 256, 0, s>>>(d_tw, d_w, n_fft, win_length);
      e = cudaGetLastError();
    }
    const int M = n_fft / 2;
    const size_t smem = sizeof(float2) * (size_t)M;
    if (e == cudaSuccess && smem > 48 * 1024)
      e = cudaFuncSetAttribute(istft_frames_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      istft_frames_kernel<<<n_frames, 256, smem, s>>>(d_S, n_frames, n_fft, ilog2(M), d_tw, d_w, d_fr);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      long long g = (out_len + 255) / 256;
      if (g > 148 * 16) g = 148 * 16;
      istft_ola_kernel<<<(unsigned)g, 256, 0, s>>>(d_fr, d_w, n_frames, n_fft, hop_length, expected, trim, out_len,
                                                   d_out);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(ws->host, d_out, out_b, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      free(res);
      cudaGetLastError();
      return cuda_status(e);
    }
    memcpy(res, ws->host, out_b);
  }
  out->data = res;
  out->shape[0] = out_len;
  out->count = out_len;
  return MM_OK;
}

}  // extern "C"
