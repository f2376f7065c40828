// Device helpers shared by the frame kernels: max encoding, vDSP-style
// threshold, power transform, padding, clip descriptors and the packed mel
// dot product.
#pragma once
#include <math.h>
#include <string.h>

#include "fft_radix.cuh"
#include "kernels.h"

namespace mm {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

// Order-preserving float -> uint map so atomicMax on uint is a float max.
__host__ __device__ __forceinline__ unsigned enc_f(float f) {
  unsigned b;
#ifdef __CUDA_ARCH__
  b = __float_as_uint(f);
#else
  memcpy(&b, &f, 4);
#endif
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float dec_f(unsigned u) {
  unsigned b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  return __uint_as_float(b);
}

// vDSP_vthr: x if x >= t else t (a NaN x becomes t).
__device__ __forceinline__ float vthr(float x, float t) { return x >= t ? x : t; }

// Frame epilogues' 10 log10(max(x, amin) / ref) as 10 log10(2) log2(max(x,
// amin)) - 10 log10(ref), with the hardware base-2 logarithm (__log2f,
// relative error about 2^-22: at most ~3e-5 dB down to amin 1e-10, far inside
// the 1e-3 dB bar).  ref_db = 10 log10(ref), computed once per launch.
__device__ __forceinline__ float db10_frame(float x, float amin, float ref_db) {
  return fmaf(3.0102999566398120f, __log2f(vthr(x, amin)), -ref_db);
}

// |X|^power from |X|^2: PW 0 -> |X|^2, 1 -> |X|, 2 -> |X|^power.
template <int PW>
__device__ __forceinline__ float apply_power(float pw, float power) {
  if constexpr (PW == 0) return pw;
  else if constexpr (PW == 1) return sqrtf(pw);
  else return powf(sqrtf(pw), power);
}

__device__ __forceinline__ long long reflect_idx(long long i, long long L) {
  if (L <= 1) return 0;
  long long period = 2 * (L - 1);
  long long m = i % period;
  if (m < 0) m += period;
  return m < L ? m : period - m;
}

__device__ __forceinline__ float sample_at(const float *sig, long long i, long long L, int pad_mode) {
  if (i >= 0 && i < L) return __ldg(sig + i);
  if (pad_mode == PAD_REFLECT) return __ldg(sig + reflect_idx(i, L));
  return 0.0f;
}

__device__ __forceinline__ int padx(int i) { return i + (i >> 4); }

__device__ __forceinline__ ClipDesc load_clip(const ClipDesc *p) {
  ClipDesc d;
  d.sig_off = __ldg(&p->sig_off);
  d.length = __ldg(&p->length);
  d.frame_off = __ldg(&p->frame_off);
  d.out_off = __ldg(&p->out_off);
  d.n_frames = __ldg(&p->n_frames);
  d.tile_base = __ldg(&p->tile_base);
  return d;
}

__device__ __forceinline__ cpx ldc(const float2 *p) {
  float2 v = __ldg(p);
  return {v.x, v.y};
}

__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

// Barrier over the TPF threads of frame group f, returning the OR of `pred`
// over the group.  Groups of >= 32 threads use named barrier f+1; smaller
// groups live inside one warp.
template <int TPF>
__device__ __forceinline__ bool frame_sync_or(int f, bool pred) {
  if constexpr (TPF >= 32) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((unsigned)pred), "r"(f + 1), "r"(TPF)
        : "memory");
    return r != 0;
  } else {
    __syncwarp();
    const unsigned lane = threadIdx.x & 31;
    const unsigned mask = ((TPF == 32) ? 0xffffffffu : ((1u << TPF) - 1u)) << (lane & ~(unsigned)(TPF - 1));
    const unsigned b = __ballot_sync(0xffffffffu, pred);
    return (b & mask) != 0;
  }
}

template <int TPF>
__device__ __forceinline__ void frame_sync(int f) {
  if constexpr (TPF >= 32) {
    asm volatile("bar.sync %0, %1;" ::"r"(f + 1), "r"(TPF) : "memory");
  } else {
    __syncwarp();
  }
}

// Packed mel weights are staged in shared memory up to this size.
constexpr int kMelSmemMax = 12288;  // floats
// Shared-memory bytes for the mel tables: per-mel info + packed weights (when they fit).
__host__ __device__ inline size_t mel_smem_bytes(int n_mels, int nnz) {
  return 16 * (size_t)n_mels + (nnz <= kMelSmemMax ? align16(4 * (size_t)nnz) : 0);
}

// Dot product of one packed mel row with a power spectrum.
__device__ __forceinline__ float mel_dot(int4 info, const float *w, const float *P, bool bad) {
  const float *wr = w + info.z;
  const float *pr = P + info.x;
  float a0 = 0.0f, a1 = 0.0f;
  int q = 0;
  for (; q + 1 < info.y; q += 2) {
    a0 = fmaf(wr[q], pr[q], a0);
    a1 = fmaf(wr[q + 1], pr[q + 1], a1);
  }
  if (q < info.y) a0 = fmaf(wr[q], pr[q], a0);
  float acc = a0 + a1;
  if (info.w || bad) acc = __int_as_float(0x7fc00000);
  return acc;
}

}  // namespace mm
