// Features built on the spectral front end (additive to the MFCC path):
// onset strength from the log-mel rows, delta and stack_memory of feature
// matrices.
//
//   onset_kernel       OnsetDetection.onsetStrength (Rhythm/OnsetDetection.swift:23-139)
//   delta_kernel       Delta.compute (Features/Delta.swift:137-241)
//   stack_memory_kernel Delta.stackMemory (Features/Delta.swift:256-290)
#include <math.h>

#include "frame_common.cuh"
#include "kernels.h"

namespace mm {

// One warp per output frame, 8 warps per CTA, tiles of kDctTile frames of
// one clip (the DCT tile tables).  Lanes stride over the bands; the mean is a
// fixed-order warp sum.
__global__ void __launch_bounds__(256) onset_kernel(OnsetArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int ti = blockIdx.x; ti < a.total_tiles; ti += gridDim.x) {
    const int c = __ldg(a.tile_clip + ti);
    const ClipDesc cd = load_clip(a.clips + c);
    const int tf = __ldg(a.tile_first + ti);
    const int T = cd.n_frames;
    const float thr = a.top_db > 0.0f ? dec_f(__ldg(a.clip_max + c)) - a.top_db : -INFINITY;
    const int o_end = min(tf + kDctTile, T);
    for (int o = tf + warp; o < o_end; o += 8) {
      const int i = o - a.shift;
      const bool live = i >= 0 && i + a.lag < T;
      const float *cur = a.mel_db + (cd.frame_off + (live ? i + a.lag : 0)) * (long long)a.n_mels;
      const float *prev = a.mel_db + (cd.frame_off + (live ? i : 0)) * (long long)a.n_mels;
      float sum = 0.0f;
      for (int b = lane; b < a.n_mels; b += 32) {
        float d = 0.0f;
        if (live) d = fmaxf(0.0f, vthr(__ldg(cur + b), thr) - vthr(__ldg(prev + b), thr));
        if (a.bands) a.out[cd.out_off + (long long)b * T + o] = d;
        else sum += d;
      }
      if (!a.bands) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
        if (lane == 0) a.out[cd.out_off + o] = sum / (float)a.n_mels;
      }
    }
  }
}

cudaError_t launch_onset(const OnsetArgs &a, cudaStream_t s) {
  if (a.total_tiles <= 0 || a.n_mels <= 0) return cudaSuccess;
  int grid = a.total_tiles < 148 * 8 ? a.total_tiles : 148 * 8;
  onset_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// y[f][t]: the Savitzky-Golay filter over x[f][t-half .. t+half]; the first
// and last `half` frames take the filter over the first / last `width` frames.
__global__ void delta_kernel(const float *x, float *y, int n_features, int n_frames, int width, DeltaCoeffs c) {
  const long long n = (long long)n_features * n_frames;
  const int half = width / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i / n_frames), t = (int)(i - (long long)f * n_frames);
    int start = t - half;
    if (t < half) start = 0;
    else if (t >= n_frames - half) start = n_frames - width;
    const float *row = x + (long long)f * n_frames + start;
    float v = 0.0f;
    for (int k = 0; k < width; k++) v = fmaf(c.c[k], __ldg(row + k), v);
    y[i] = v;
  }
}

cudaError_t launch_delta(const float *x, float *y, int n_features, int n_frames, int width, DeltaCoeffs c,
                         cudaStream_t s) {
  const long long n = (long long)n_features * n_frames;
  if (n <= 0) return cudaSuccess;
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  delta_kernel<<<(unsigned)g, 256, 0, s>>>(x, y, n_features, n_frames, width, c);
  return cudaGetLastError();
}

__global__ void stack_memory_kernel(const float *x, float *y, int n_features, int n_frames, int n_steps,
                                    int delay) {
  const long long n = (long long)n_features * n_steps * n_frames;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / n_frames;
    const int t = (int)(i - r * n_frames);
    const int step = (int)(r / n_features), f = (int)(r - (long long)step * n_features);
    const long long src_t = (long long)t - (long long)step * delay;
    y[i] = (src_t >= 0 && src_t < n_frames) ? __ldg(x + (long long)f * n_frames + src_t) : 0.0f;
  }
}

cudaError_t launch_stack_memory(const float *x, float *y, int n_features, int n_frames, int n_steps, int delay,
                                cudaStream_t s) {
  const long long n = (long long)n_features * n_steps * n_frames;
  if (n <= 0) return cudaSuccess;
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  stack_memory_kernel<<<(unsigned)g, 256, 0, s>>>(x, y, n_features, n_frames, n_steps, delay);
  return cudaGetLastError();
}

}  // namespace mm
