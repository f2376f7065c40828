// Warp-per-frame front-end kernel (launch variant 3, n_fft 256..2048, MFCC
// path; n_fft 4096 on a warp pair, frame_warp2_kernel below): framing + periodic Hann + real FFT + |X|^2 + Slaney mel + log10 per
// frame, with a running per-clip maximum for top_db.
//
// The reference computes the same per frame on the CPU, one frame after the
// other (STFT.swift:287-335 window/FFT/power, MelSpectrogram.swift:122-138 mel,
// Scaling.swift:73-118 dB).  Here a frame is owned by TPF = n_fft/64 lanes of a
// warp; each lane holds 32 complex points of the packed sequence
// z[n] = x[2n] w[2n] + i x[2n+1] w[2n+1] (M = n_fft/2 points):
//
//   n = j + TPF r   (j = lane in the frame group, r = register)
//   k = k1 + 32 k2
//   stage 1: 32-point DFT over r in registers       -> Y[j][k1]
//            twiddle W_M^(j k1)
//   one shared-memory transpose (row stride 33, conflict-free; one frame per
//   warp: stored transposed with stride 34 and read back as float4)
//   stage 2: TPF-point DFTs over j in registers      -> Z[k1 + 32 k2]
//   real split X[k] = E + W_N^k O, X[M-k] = conj(E - W_N^k O), both from the
//   pair (Z[k], Z[M-k]): the stage-2 columns are dealt to lanes so that k1
//   and 32-k1 sit in the same lane (TPF < 32); for TPF = 32 the partner lanes
//   l and 32-l swap the upper 16 registers by shuffle and each takes 16 pairs.
//
// Only warp-level synchronisation is used.  The window is staged in shared
// memory halved (exact in binary floating point), so the real split's
// E + W O, formed without its factor 1/2, is X itself and the spectrum is
// |X|^2, bit for bit the values of the unscaled transform divided by 4: a bin
// overflows float32 only where the reference's |X|^2 does.  The window, the
// stage-2 twiddles and the mel tables are staged once per CTA.
#include <math.h>

#include <algorithm>
#include <type_traits>

#include <cuda_fp16.h>

#include "async_copy.cuh"
#include "fft_radix.cuh"
#include "frame_common.cuh"
#include "kernels.h"
#include "tcgen05.cuh"

namespace mm {

// ---------------------------------------------------------------------------
// compile-time cos / sin of 2 pi k / d: octant reduction, then Taylor series
// in double (|x| <= pi/4, 12 terms: error far below float rounding)
// ---------------------------------------------------------------------------
constexpr double kPiD = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double ce_sin_q(double x) {
  double term = x, sum = x;
  for (int n = 1; n < 12; n++) {
    term *= -x * x / (double)((2 * n) * (2 * n + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double ce_cos_q(double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 12; n++) {
    term *= -x * x / (double)((2 * n - 1) * (2 * n));
    sum += term;
  }
  return sum;
}
// which = 0: cos(2 pi k / d), 1: sin(2 pi k / d)
__host__ __device__ constexpr double ce_trig(long long k, long long d, int which) {
  k %= d;
  if (k < 0) k += d;
  const long long q = (8 * k) / d;                                   // octant 0..7
  const double phi = kPiD * (double)(8 * k - q * d) / (4.0 * (double)d);  // in [0, pi/4)
  const double psi = kPiD * (double)(d * (q + 1) - 8 * k) / (4.0 * (double)d);  // pi/4 - phi
  double c = 0.0, s = 0.0;
  switch (q) {
    case 0: c = ce_cos_q(phi); s = ce_sin_q(phi); break;
    case 1: c = ce_sin_q(psi); s = ce_cos_q(psi); break;
    case 2: c = -ce_sin_q(phi); s = ce_cos_q(phi); break;
    case 3: c = -ce_cos_q(psi); s = ce_sin_q(psi); break;
    case 4: c = -ce_cos_q(phi); s = -ce_sin_q(phi); break;
    case 5: c = -ce_sin_q(psi); s = -ce_cos_q(psi); break;
    case 6: c = ce_sin_q(phi); s = -ce_cos_q(phi); break;
    default: c = ce_cos_q(psi); s = -ce_sin_q(psi); break;
  }
  return which == 0 ? c : s;
}

template <int I, int N, typename Fn>
__device__ __forceinline__ void static_for(Fn &&fn) {
  if constexpr (I < N) {
    fn(std::integral_constant<int, I>{});
    static_for<I + 1, N>(fn);
  }
}

// a * exp(-2 pi i K / D), with the exact special angles spelled out.
template <int K, int D>
__device__ __forceinline__ cpx tw_const(cpx a) {
  constexpr int k = ((K % D) + D) % D;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (4 * k == D) {
    return mul_mi(a);
  } else if constexpr (2 * k == D) {
    return {-a.x, -a.y};
  } else if constexpr (4 * k == 3 * D) {
    return mul_pi(a);
  } else if constexpr (8 * k == D) {
    return mul_w8_1(a);
  } else if constexpr (8 * k == 3 * D) {
    return mul_w8_3(a);
  } else if constexpr (8 * k == 5 * D) {
    return {-kR * (a.x + a.y), kR * (a.x - a.y)};
  } else if constexpr (8 * k == 7 * D) {
    return {kR * (a.x - a.y), kR * (a.x + a.y)};
  } else {
    constexpr float c = (float)ce_trig(k, D, 0);
    constexpr float s = -(float)ce_trig(k, D, 1);
    return {fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c)};
  }
}

// In-place 32-point DFT, natural order: radix-2 decimation in time over two
// 16-point DFTs.
__device__ __forceinline__ void dft32(cpx *v) {
  cpx e[16], o[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    e[m] = v[2 * m];
    o[m] = v[2 * m + 1];
  }
  dft16(e);
  dft16(o);
  static_for<0, 16>([&](auto ki) {
    constexpr int k = decltype(ki)::value;
    const cpx t = tw_const<k, 32>(o[k]);
    v[k] = cadd(e[k], t);
    v[k + 16] = csub(e[k], t);
  });
}

template <int R>
__device__ __forceinline__ void dft_any(cpx *v) {
  if constexpr (R == 32) dft32(v);
  else dft<R>(v);
}

// W_N^s for any s >= 0 from the quarter table q[t] = W_N^t, t < N/4.
__device__ __forceinline__ cpx root_q(const float2 *q, int s, int N) {
  s &= N - 1;
  const int quarter = N >> 2;
  const int h = s / quarter, r = s - h * quarter;
  const float2 w = __ldg(q + r);
  switch (h) {
    case 0: return {w.x, w.y};
    case 1: return {w.y, -w.x};   // * (-i)
    case 2: return {-w.x, -w.y};  // * (-1)
    default: return {-w.y, w.x};  // * (+i)
  }
}

// Samples (x[i], x[i+1]) for i = first + stride r, r < 32, with the padding
// rule of sample_at; used only for frames that overlap the clip's edges.
__device__ __noinline__ void gather_edge(cpx *out, const float *sig, long long first, long long length,
                                         int pad_mode, int stride) {
  for (int r = 0; r < 32; r++) {
    const long long n0 = first + (long long)stride * r;
    out[r] = {sample_at(sig, n0, length, pad_mode), sample_at(sig, n0 + 1, length, pad_mode)};
  }
}

template <int LOG2N>
struct WShape {
  static constexpr int N = 1 << LOG2N;
  static constexpr int M = N / 2;
  static constexpr int TPF = M / 32;     // lanes per frame
  static constexpr int FPW = 32 / TPF;   // frames per warp
  static constexpr int C = FPW;          // stage-2 columns per lane
  static constexpr int HALF = C / 2;
  // complex slots per frame buffer: TPF rows of 33 (one frame per warp: the
  // stage-1 results stored transposed, 32 columns of 34)
  static constexpr int FSTRIDE = TPF == 32 ? 32 * 34 : TPF * 33;
  static constexpr int NW = 8;              // warps per CTA
  static constexpr int THREADS = 32 * NW;
  static constexpr int F = NW * FPW;        // frames per CTA tile
  static_assert(TPF >= 4 && TPF <= 32, "n_fft must be 256..2048");
};

// Real-split twiddles W_N^(l + 32 i), i < 16, of lane l (one frame per warp
// only): 512 complex, staged as pairs (i = 2p, 2p + 1) in float4 [32 p + l].
template <int LOG2N>
__host__ __device__ constexpr size_t warp_split_tw() {
  return WShape<LOG2N>::C == 1 ? size_t(16 * 32) * 8 : 0;
}

template <int LOG2N>
__host__ __device__ constexpr size_t warp_fixed_smem() {
  using S = WShape<LOG2N>;
  return size_t(8) * S::TPF * 16 + align16(size_t(S::N) * 4) + warp_split_tw<LOG2N>() +
         size_t(S::F) * S::FSTRIDE * 8;
}

int warp_frames_per_tile(int log2n) {
  switch (log2n) {
    case 8: return WShape<8>::F;
    case 9: return WShape<9>::F;
    case 10: return WShape<10>::F;
    case 11: return WShape<11>::F;
    case 12: return 8;  // frame_warp2_kernel: one frame per warp pair, 16 warps
    default: return 0;
  }
}

// Position of bin k in the padded power spectrum: PS floats per 32 bins,
// k + (PS - 32) min(k / 32, TPF - 1).
template <int TPF, int PS = 33>
__device__ __forceinline__ int pad_bin(int k) {
  const int q = k >> 5;
  return k + (PS - 32) * (q < TPF - 1 ? q : TPF - 1);
}

// mel_dot over the padded power spectrum.
template <int TPF, int PS = 33>
__device__ __forceinline__ float mel_dot_pad(int4 info, const float *w, const float *P, bool bad) {
  const float *wr = w + info.z;
  float acc = 0.0f;
  for (int q = 0; q < info.y; q++) acc = fmaf(wr[q], P[pad_bin<TPF, PS>(info.x + q)], acc);
  if (info.w || bad) acc = __int_as_float(0x7fc00000);
  return acc;
}

// stage-2 column of slot c for lane l (see the header comment)
template <int TPF, int C, int c>
__device__ __forceinline__ int stage2_col(int l) {
  if constexpr (C == 1) {
    return l;
  } else if constexpr (c < C / 2) {
    return l + TPF * c;
  } else if constexpr (c == C / 2) {
    return l == 0 ? 16 : 32 - l;
  } else {
    return 32 - l - TPF * (c - C / 2);
  }
}

template <int LOG2N>
__global__ void __launch_bounds__(WShape<LOG2N>::THREADS, 2) frame_warp_kernel(FrontArgs a) {
  using S = WShape<LOG2N>;
  constexpr int N = S::N, M = S::M, TPF = S::TPF, C = S::C, HALF = S::HALF, F = S::F;
  // floats per 32 bins of the padded power spectrum: 36 for one frame per
  // warp, so that a lane's 32 bins are 16-byte aligned and read as float4
  constexpr int PS = (TPF == 32) ? 36 : 33;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nmel = a.n_mels;
  const float ref_db = 10.0f * log10f(a.ref);
  // Lane walk over the per-bin split of the filterbank (else packed rows).
  const bool lanes = a.mel_lane_ok != 0;
  const bool mel_in_smem = a.mel_nnz <= kMelSmemMax;
  unsigned char *sp = smem;
  // stage-1 twiddles as pairs: tw4[p][j] = (W_M^(j (2p+1)), W_M^(j (2p+2))), p < 8
  float4 *tw4 = reinterpret_cast<float4 *>(sp);
  sp += size_t(8) * TPF * 16;
  // analysis window (halved), the sample pairs of registers r, r + 1 of lane
  // l as one float4 at [r / 2][l]
  float4 *win_s = reinterpret_cast<float4 *>(sp);
  sp += align16(size_t(N) * 4);
  float4 *rs_tw = reinterpret_cast<float4 *>(sp);  // C == 1: real-split twiddle pairs [32 p + l]
  sp += warp_split_tw<LOG2N>();
  cpx *bufs = reinterpret_cast<cpx *>(sp);
  sp += size_t(F) * S::FSTRIDE * 8;
  // lanes: band words, lane words, lane-minor weights (bins 2p, 2p + 1 of
  // lane l as one float4 at [p][l], p < 17); else packed rows
  int *band_s = reinterpret_cast<int *>(sp);
  int2 *lane_s = reinterpret_cast<int2 *>(sp + align16(4 * (size_t)nmel));
  float4 *lw_s = reinterpret_cast<float4 *>(sp + align16(4 * (size_t)nmel) + 8 * TPF);
  int4 *mel_s = reinterpret_cast<int4 *>(sp);
  float *melw_s = reinterpret_cast<float *>(sp + 16 * (size_t)nmel);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = lane / TPF;       // frame of this lane within the warp
  const int l = lane - grp * TPF;   // lane within the frame group
  const float2 *twq = a.tw_split;   // W_N^t, t < N/4

  for (int i = tid; i < 8 * TPF; i += S::THREADS) {
    const int p = i / TPF, j = i - p * TPF;
    const cpx u = root_q(twq, 2 * j * (2 * p + 1), N), w = root_q(twq, 2 * j * (2 * p + 2), N);
    tw4[i] = make_float4(u.x, u.y, w.x, w.y);
  }
  for (int i = tid; i < 16 * TPF; i += S::THREADS) {  // halved: see the header comment
    const int p = i / TPF, j = i - p * TPF;
    const float2 u = __ldg(reinterpret_cast<const float2 *>(a.window) + j + TPF * (2 * p));
    const float2 w = __ldg(reinterpret_cast<const float2 *>(a.window) + j + TPF * (2 * p + 1));
    win_s[i] = make_float4(0.5f * u.x, 0.5f * u.y, 0.5f * w.x, 0.5f * w.y);
  }
  if constexpr (C == 1)
    for (int i = tid; i < 8 * 32; i += S::THREADS) {
      const int p = i >> 5, ll = i & 31;
      const cpx u = root_q(twq, ll + 64 * p, N), w = root_q(twq, ll + 32 * (2 * p + 1), N);
      rs_tw[i] = make_float4(u.x, u.y, w.x, w.y);
    }
  if (lanes) {
    for (int i = tid; i < nmel; i += S::THREADS) band_s[i] = __ldg(a.mel_band + i);
    for (int i = tid; i < TPF; i += S::THREADS) lane_s[i] = __ldg(a.mel_lane + i);
    for (int i = tid; i < 17 * TPF; i += S::THREADS) {
      const int p = i / TPF, j = i - p * TPF;
      const float2 u = __ldg(a.mel_lw + 2 * p * TPF + j);
      const float2 w = 2 * p + 1 < 33 ? __ldg(a.mel_lw + (2 * p + 1) * TPF + j) : make_float2(0.0f, 0.0f);
      lw_s[i] = make_float4(u.x, u.y, w.x, w.y);
    }
  } else {
    for (int i = tid; i < nmel; i += S::THREADS) mel_s[i] = __ldg(a.mel_info + i);
    if (mel_in_smem)
      for (int i = tid; i < a.mel_nnz; i += S::THREADS) melw_s[i] = __ldg(a.mel_pw + i);
  }
  const float *melw = mel_in_smem ? melw_s : a.mel_pw;
  __syncthreads();

  // real-split bases W_N^(first bin of each column pair)
  cpx base_c[HALF > 0 ? HALF : 1];
  cpx base_hi;
  if constexpr (C == 1) {
    base_c[0] = root_q(twq, l, N);
    base_hi = base_c[0];
  } else {
#pragma unroll
    for (int c = 0; c < HALF; c++) base_c[c] = root_q(twq, l + TPF * c, N);
    base_hi = (l == 0) ? root_q(twq, 16 + 3 * (N / 4), N) : base_c[0];
  }

  cpx *fb = bufs + (warp * S::FPW + grp) * S::FSTRIDE;
  // power spectrum, padded: bin k at k + (PS - 32) min(k / 32, TPF - 1), so
  // that lane l of the group reads its bins [32 l, 32 l + 32) at PS l + b, and
  // the Nyquist bin M at PS (TPF - 1) + 32; group g starts TPF g floats into
  // its buffer so that the groups of a warp fall in disjoint banks
  float *P = reinterpret_cast<float *>(fb) + TPF * grp;
  const unsigned gmask = (TPF == 32) ? FULL : (((1u << TPF) - 1u) << (grp * TPF));

  const int total = a.total_tiles;
  const int t_begin = (int)((long long)blockIdx.x * total / gridDim.x);
  const int t_end = (int)((long long)(blockIdx.x + 1) * total / gridDim.x);
  int cur = -1;
  float vmax = -INFINITY;

  for (int tile = t_begin; tile < t_end; tile++) {
    const int c = __ldg(a.tile_clip + tile);
    if (c != cur) {  // warp-uniform: every frame of a tile belongs to one clip
      float m = vmax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
      if (lane == 0 && cur >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur, enc_f(m));
      cur = c;
      vmax = -INFINITY;
    }
    const ClipDesc cd = load_clip(a.clips + c);
    const int t = (tile - cd.tile_base) * F + warp * S::FPW + grp;
    if constexpr (TPF == 32) {
      if (t >= cd.n_frames) continue;  // warp-uniform
    }
    const bool valid = t < cd.n_frames;
    const long long s0 = (long long)t * a.hop - a.pad;
    const float *sig = a.signal + cd.sig_off;

    // ---- gather: v[r] = (x[2n], x[2n+1]) for n = l + TPF r
    cpx v[32];
    if (s0 >= 0 && s0 + N <= cd.length) {
      const float *base = sig + s0 + 2 * l;
      if (((cd.sig_off + s0) & 1) == 0) {
#pragma unroll
        for (int r = 0; r < 32; r++) {
          const float2 x = __ldg(reinterpret_cast<const float2 *>(base + 2 * TPF * r));
          v[r] = {x.x, x.y};
        }
      } else {
#pragma unroll
        for (int r = 0; r < 32; r++) v[r] = {__ldg(base + 2 * TPF * r), __ldg(base + 2 * TPF * r + 1)};
      }
    } else {
      // frames that reach into the padding (a few per clip): out of line, so
      // that their index arithmetic does not weigh on the interior path
      cpx tmp[32];
      gather_edge(tmp, sig, s0 + 2 * l, cd.length, a.pad_mode, 2 * TPF);
#pragma unroll
      for (int r = 0; r < 32; r++) v[r] = tmp[r];
    }
    // ---- window
    {
      const float4 *wb = win_s + l;
#pragma unroll
      for (int r = 0; r < 32; r += 2) {
        const float4 w = wb[TPF * (r / 2)];
        v[r].x *= w.x;
        v[r].y *= w.y;
        v[r + 1].x *= w.z;
        v[r + 1].y *= w.w;
      }
    }

    // ---- stage 1: 32-point DFT over registers; its last butterflies are
    // followed directly by the twiddle W_M^(l k1) and the store into row l of
    // the frame buffer (stride 33; one frame per warp: into column l of rows
    // of 34, so that stage 2 reads its column as float4), so that registers
    // free up as it goes.
    __syncwarp();  // the previous frame's mel reads of P are done
    {
      cpx e[16], o[16];
#pragma unroll
      for (int m = 0; m < 16; m++) {
        e[m] = v[2 * m];
        o[m] = v[2 * m + 1];
      }
      dft16(e);
      dft16(o);
      cpx *row = fb + l * 33;
      // W_M^(l (k + 16)) = W_M^(l k) W_M^(16 l): half of the table reads
      const float4 t78 = tw4[7 * TPF + l];  // k = 15, 16
      const cpx g16 = {t78.z, t78.w};
      float4 tp = t78;
      static_for<0, 16>([&](auto ki) {
        constexpr int k = decltype(ki)::value;
        const cpx t = tw_const<k, 32>(o[k]);
        cpx lo = cadd(e[k], t), hi = csub(e[k], t);
        if constexpr (k > 0) {
          // pair k / 2 holds k (odd) and k + 1
          if constexpr (k == 15) tp = t78;
          else if constexpr (k % 2 == 1) tp = tw4[(k / 2) * TPF + l];
          const cpx tk = (k % 2 == 1) ? cpx{tp.x, tp.y} : cpx{tp.z, tp.w};
          lo = cmul(lo, tk);
          hi = cmul(hi, cmul(tk, g16));
        } else {
          hi = cmul(hi, g16);
        }
        if constexpr (C == 1) {
          fb[k * 34 + l] = lo;
          fb[(k + 16) * 34 + l] = hi;
        } else {
          row[k] = lo;
          row[k + 16] = hi;
        }
      });
    }
    __syncwarp();
    if constexpr (C == 1) {  // column l: Y[jj][l] at 34 l + jj
      const float4 *colp = reinterpret_cast<const float4 *>(fb + 34 * l);
#pragma unroll
      for (int jj = 0; jj < 32; jj += 2) {
        const float4 y = colp[jj / 2];
        v[jj] = {y.x, y.y};
        v[jj + 1] = {y.z, y.w};
      }
    } else {
      static_for<0, C>([&](auto ci) {
        constexpr int cc = decltype(ci)::value;
        const int col = stage2_col<TPF, C, cc>(l);
#pragma unroll
        for (int jj = 0; jj < TPF; jj++) v[cc * TPF + jj] = fb[jj * 33 + col];
      });
    }
    // ---- stage 2: TPF-point DFTs, v[c*TPF + k2] = Z[col(c) + 32 k2]
#pragma unroll
    for (int cc = 0; cc < C; cc++) dft_any<TPF>(v + cc * TPF);
    __syncwarp();  // every lane has read its columns: fb becomes P

    // ---- real split, P[k] = |X[k]|^2 (the window was halved)
    if constexpr (C == 1) {
      // lanes l and 32-l swap registers 16..31: pair i of lane l is
      // (Z[l + 32 i], Z[M - l - 32 i]) = (v[i], partner's v[31 - i]); lane 0
      // pairs with itself: (v[i], v[32 - i]) and the self pair v[16] (k = M/2).
      const int src = (32 - l) & 31;
      cpx rcv[16];
#pragma unroll
      for (int m = 0; m < 16; m++) {
        rcv[m].x = __shfl_sync(FULL, v[16 + m].x, src);
        rcv[m].y = __shfl_sync(FULL, v[16 + m].y, src);
      }
      const bool l0 = (l == 0);
      float *Pa = P + l;  // bin l + 32 i at l + PS i
      float4 rsp;
      // bin M - l - 32 i at M + (PS - 32)(TPF - 1) - l - PS i (lane 0, i > 0:
      // PS - 32 further on; its i = 0 is the Nyquist bin)
      float *Pb = P + (M + (PS - 32) * (TPF - 1) - l) + (l0 ? PS - 32 : 0);
      static_for<0, 16>([&](auto ki) {
        constexpr int i = decltype(ki)::value;
        const cpx za = v[i];
        cpx zb;
        if constexpr (i == 0) zb = l0 ? v[0] : rcv[15];
        else zb = l0 ? rcv[16 - i] : rcv[15 - i];
        const float ex = za.x + zb.x, ey = za.y - zb.y;
        const float ox = za.y + zb.y, oy = zb.x - za.x;
        if constexpr (i % 2 == 0) rsp = rs_tw[32 * (i / 2) + l];
        const cpx w = (i % 2 == 0) ? cpx{rsp.x, rsp.y} : cpx{rsp.z, rsp.w};  // W_N^(l + 32 i)
        const float wr = fmaf(w.x, ox, -w.y * oy), wi = fmaf(w.x, oy, w.y * ox);
        const float xr = ex + wr, xi = ey + wi;
        const float yr = ex - wr, yi = ey - wi;
        const float p = fmaf(xr, xr, xi * xi), q = fmaf(yr, yr, yi * yi);
        Pa[PS * i] = p;
        if constexpr (i == 0) Pb[l0 ? -(PS - 32) : 0] = q;  // lane 0: the Nyquist bin
        else Pb[-PS * i] = q;
      });
      if (l0) P[M / 2 + (PS - 32) * (TPF / 2)] = 4.0f * fmaf(rcv[0].x, rcv[0].x, rcv[0].y * rcv[0].y);
    } else {
      const bool l0 = (l == 0);
      static_for<0, HALF>([&](auto ci) {
        constexpr int cc = decltype(ci)::value;
        static_for<0, TPF>([&](auto ki) {
          constexpr int k2 = decltype(ki)::value;
          cpx za, zb, base;
          int ka;
          if constexpr (cc == 0) {
            constexpr bool lo = k2 < TPF / 2;
            constexpr int ia0 = lo ? k2 : HALF * TPF + (k2 - TPF / 2);
            constexpr int ib0 = lo ? (TPF - k2) % TPF : HALF * TPF + TPF - 1 - (k2 - TPF / 2);
            constexpr int ia = k2, ib = HALF * TPF + TPF - 1 - k2;
            za = l0 ? v[ia0] : v[ia];
            zb = l0 ? v[ib0] : v[ib];
            base = lo ? base_c[0] : base_hi;
            ka = l0 ? (lo ? 32 * k2 : 16 + 32 * (k2 - TPF / 2)) : l + 32 * k2;
          } else {
            za = v[cc * TPF + k2];
            zb = v[(cc + HALF) * TPF + TPF - 1 - k2];
            base = base_c[cc];
            ka = l + TPF * cc + 32 * k2;
          }
          const float ex = za.x + zb.x, ey = za.y - zb.y;
          const float ox = za.y + zb.y, oy = zb.x - za.x;
          const cpx w = tw_const<k2, 2 * TPF>(base);
          const float wr = fmaf(w.x, ox, -w.y * oy), wi = fmaf(w.x, oy, w.y * ox);
          const float xr = ex + wr, xi = ey + wi;
          const float yr = ex - wr, yi = ey - wi;
          const float p = fmaf(xr, xr, xi * xi), q = fmaf(yr, yr, yi * yi);
          if constexpr (cc == 0) {
            P[l0 ? pad_bin<TPF>(ka) : ka + k2] = p;
            P[l0 ? pad_bin<TPF>(M - ka) : M - ka + TPF - 1 - k2] = q;
          } else {
            // l + TPF cc + 32 k2 with 0 < l + TPF cc < 32: row k2 and row TPF - 1 - k2
            P[ka + k2] = p;
            P[M - ka + TPF - 1 - k2] = q;
          }
        });
      });
      if (l0) {
        const cpx zm = v[TPF / 2];
        P[M / 2 + TPF / 2] = 4.0f * fmaf(zm.x, zm.x, zm.y * zm.y);
      }
    }
    __syncwarp();  // P complete

    // ---- log-mel row of this frame + running clip max
    float *dst = a.out + (cd.frame_off + t) * (long long)nmel;
    if (lanes) {
      // lane l sums its 32 bins (the last lane also the Nyquist bin) into
      // (R, F) = (w.x P, w.y P) and stores the pair in the next part slot at
      // every segment end; the lane holding a segment's head then adds the
      // parts of the lanes the segment runs into, and band m is the head of
      // segment m (.x) plus the head of segment m + 1 (.y).
      float2 *parts = reinterpret_cast<float2 *>(P + PS * TPF);
      const int2 li = lane_s[l];
      const unsigned fl = (unsigned)li.x;
      int slot = li.y & 1023;
      const float *pl = P + PS * l;
      const float4 *wl = lw_s + l;
      // The frame's non-finite check: `tot` accumulates p * 0 over the lane's
      // bins (NaN for a NaN or inf bin, and no overflow), then a ballot.
      float R = 0.0f, Fs = 0.0f, tot = 0.0f;
      float4 wq, pq;
#pragma unroll
      for (int b = 0; b < 32; b++) {
        float p;
        if constexpr (PS % 4 == 0) {  // four bins per load
          if ((b & 3) == 0) pq = reinterpret_cast<const float4 *>(pl)[b >> 2];
          p = (b & 3) == 0 ? pq.x : (b & 3) == 1 ? pq.y : (b & 3) == 2 ? pq.z : pq.w;
        } else {
          p = pl[b];
        }
        if ((b & 1) == 0) wq = wl[(b >> 1) * TPF];
        const float2 w = (b & 1) ? make_float2(wq.z, wq.w) : make_float2(wq.x, wq.y);
        tot = fmaf(p, 0.0f, tot);
        R = fmaf(w.x, p, R);
        Fs = fmaf(w.y, p, Fs);
        if (fl & (1u << b)) {
          parts[slot++] = make_float2(R, Fs);
          R = 0.0f;
          Fs = 0.0f;
        }
      }
      if (l == TPF - 1) {
        const float p = pl[32];
        const float4 wn = wl[16 * TPF];
        const float2 w = make_float2(wn.x, wn.y);
        tot = fmaf(p, 0.0f, tot);
        R = fmaf(w.x, p, R);
        Fs = fmaf(w.y, p, Fs);
        parts[slot] = make_float2(R, Fs);
      }
      const bool bad = (__ballot_sync(FULL, !isfinite(tot)) & gmask) != 0;
      if (l == 0) parts[li.y >> 16] = make_float2(0.0f, 0.0f);  // the empty segments' slot
      __syncwarp();
      // fix-up: this lane's last part heads a segment that runs into the next k lanes
      const int kc = (li.y >> 10) & 63;
      if (kc) {
        const int h = l == TPF - 1 ? slot : slot - 1;
        float2 hv = parts[h];
        for (int j = 1; j <= kc; j++) {
          const float2 pv = parts[h + j];
          hv.x += pv.x;
          hv.y += pv.y;
        }
        parts[h] = hv;
      }
      __syncwarp();
      for (int m = l; m < nmel; m += TPF) {
        const int bw = band_s[m];
        float acc = parts[bw & 4095].x + parts[(bw >> 12) & 4095].y;
        if (((bw >> 24) & 1) || bad) acc = __int_as_float(0x7fc00000);
        const float val = db10_frame(acc, a.amin, ref_db);
        if (valid) {
          dst[m] = val;
          vmax = fmaxf(vmax, val);
        }
      }
    } else {
      float chk = 0.0f;  // the frame's non-finite check: this lane's share of the bins, times 0
      for (int k = l; k <= M; k += TPF) chk = fmaf(P[pad_bin<TPF, PS>(k)], 0.0f, chk);
      const bool bad = (__ballot_sync(FULL, !isfinite(chk)) & gmask) != 0;
      for (int m = l; m < nmel; m += TPF) {
        const float acc = mel_dot_pad<TPF, PS>(mel_s[m], melw, P, bad);
        const float val = db10_frame(acc, a.amin, ref_db);
        if (valid) {
          dst[m] = val;
          vmax = fmaxf(vmax, val);
        }
      }
    }
  }
  float m = vmax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
  if (lane == 0 && cur >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur, enc_f(m));
}

// ---------------------------------------------------------------------------
// n_fft 4096: one frame per pair of warps (64 threads), same per-frame work.
//
//   n = j + 64 r (j < 64: thread of the pair, r < 32), k = k1 + 32 k2 (k2 < 64)
//   stage 1: 32-point DFT over r in registers, twiddle W_M^(j k1), row j of
//            the frame buffer (stride 33)
//   stage 2: the 64-point DFT over j of column k1 as 2 x 32: thread (k1, j0)
//            takes rows j0 + 2 j1 (j1 < 32) through a 32-point DFT -> A_j0[q];
//            the two threads of a column (lanes 2i, 2i+1) swap half of their
//            outputs by shuffle, and thread j0 forms
//            Z[k1 + 32 q] = A_0[q] + W_64^q A_1[q] and
//            Z[k1 + 32 (q + 32)] = A_0[q] - W_64^q A_1[q] for q = 2 i + j0.
//   Even columns live in the pair's first warp, odd ones in its second
//   (lane = 2 (k1 >> 1) + j0), so the real-split partner (32 - k1, 1 - j0)
//   of a thread sits in its warp; the two swap their upper 16 registers as
//   in the single-warp kernel.  Column 0 pairs inside each thread.
// Every shared-memory pattern (row stores, column loads, twiddles, spectrum
// stores, the walk) is conflict-free for this lane assignment.
// ---------------------------------------------------------------------------
struct W2Shape {
  static constexpr int N = 4096;
  static constexpr int M = N / 2;
  static constexpr int TPF = 64;            // threads per frame
  static constexpr int FSTRIDE = TPF * 33;  // complex slots per frame buffer
  static constexpr int NW = 16;             // warps per CTA (one CTA per SM)
  static constexpr int THREADS = 32 * NW;
  static constexpr int F = NW / 2;          // frames per CTA tile
  static constexpr int RS = 33 * 32;        // real-split twiddles W_N^(c + 32 s) at 33 s + c
  static constexpr int MEL_SMEM_MAX = 8192; // packed weights staged up to this many floats
};

__host__ __device__ constexpr size_t warp2_fixed_smem() {
  using S = W2Shape;
  return size_t(8) * S::TPF * 16 + align16(size_t(S::N) * 4) + align16(size_t(S::RS) * 8) +
         size_t(S::F) * S::FSTRIDE * 8;
}

__global__ void __launch_bounds__(W2Shape::THREADS, 1) frame_warp2_kernel(FrontArgs a) {
  using S = W2Shape;
  constexpr int N = S::N, M = S::M, TPF = S::TPF, F = S::F;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nmel = a.n_mels;
  const float ref_db = 10.0f * log10f(a.ref);
  const bool lanes = a.mel_lane_ok != 0;
  const bool mel_in_smem = a.mel_nnz <= S::MEL_SMEM_MAX;
  unsigned char *sp = smem;
  // The tables a thread reads once per frame are staged as float4 pairs of
  // the entries it reads in turn (half the load instructions, same bytes):
  // stage-1 twiddles tw4[p][j] = (W_M^(j (2p+1)), W_M^(j (2p+2))), p < 8
  float4 *tw4 = reinterpret_cast<float4 *>(sp);
  sp += size_t(8) * TPF * 16;
  // the halved window: samples of registers r, r + 1 of thread j at [r / 2][j]
  float4 *win_s = reinterpret_cast<float4 *>(sp);
  sp += align16(size_t(N) * 4);
  // real-split twiddles: row 2p + j0, column c holds (W_N^(c + 32 (4p + j0)),
  // W_N^(c + 32 (4p + 2 + j0))), rows of 33 (conflict-free)
  float4 *rs_tw = reinterpret_cast<float4 *>(sp);
  sp += align16(size_t(S::RS) * 8);
  cpx *bufs = reinterpret_cast<cpx *>(sp);
  sp += size_t(F) * S::FSTRIDE * 8;
  // lanes: band words, lane words, lane-minor weights; else packed weights
  // (the packed rows' descriptors are read from global memory)
  int *band_s = reinterpret_cast<int *>(sp);
  int2 *lane_s = reinterpret_cast<int2 *>(sp + align16(4 * (size_t)nmel));
  float4 *lw_s = reinterpret_cast<float4 *>(sp + align16(4 * (size_t)nmel) + 8 * TPF);  // weight pairs [p][j]
  float *melw_s = reinterpret_cast<float *>(sp);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int fp = warp >> 1;              // frame of this warp pair within the tile
  const int half = warp & 1;             // 0: even columns, 1: odd columns
  const int j = half * 32 + lane;        // stage-1 row, walk lane
  const int j0 = lane & 1;               // stage-2 half of the column
  const int col = 2 * (lane >> 1) + half;  // stage-2 column k1
  const bool c0 = col == 0;
  const int partner = 2 * (half ? 15 - (lane >> 1) : (16 - (lane >> 1)) & 15) + (1 - j0);
  const float2 *twq = a.tw_split;  // W_N^t, t < N/4

  for (int i = tid; i < 8 * TPF; i += S::THREADS) {
    const int p = i / TPF, jj = i - p * TPF;
    const cpx u = root_q(twq, 2 * jj * (2 * p + 1), N), w = root_q(twq, 2 * jj * (2 * p + 2), N);
    tw4[i] = make_float4(u.x, u.y, w.x, w.y);
  }
  for (int i = tid; i < 16 * TPF; i += S::THREADS) {  // halved: see the header comment
    const int p = i / TPF, jj = i - p * TPF;
    const float2 u = __ldg(reinterpret_cast<const float2 *>(a.window) + jj + TPF * (2 * p));
    const float2 w = __ldg(reinterpret_cast<const float2 *>(a.window) + jj + TPF * (2 * p + 1));
    win_s[i] = make_float4(0.5f * u.x, 0.5f * u.y, 0.5f * w.x, 0.5f * w.y);
  }
  for (int i = tid; i < 16 * 33; i += S::THREADS) {
    const int row = i / 33, cc = i - 33 * row, p = row >> 1, jj0 = row & 1;
    if (cc < 32) {
      const cpx u = root_q(twq, cc + 32 * (4 * p + jj0), N), w = root_q(twq, cc + 32 * (4 * p + 2 + jj0), N);
      rs_tw[i] = make_float4(u.x, u.y, w.x, w.y);
    } else {
      rs_tw[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
  if (lanes) {
    for (int i = tid; i < nmel; i += S::THREADS) band_s[i] = __ldg(a.mel_band + i);
    for (int i = tid; i < TPF; i += S::THREADS) lane_s[i] = __ldg(a.mel_lane + i);
    for (int i = tid; i < 17 * TPF; i += S::THREADS) {
      const int p = i / TPF, jj = i - p * TPF;
      const float2 u = __ldg(a.mel_lw + 2 * p * TPF + jj);
      const float2 w = 2 * p + 1 < 33 ? __ldg(a.mel_lw + (2 * p + 1) * TPF + jj) : make_float2(0.0f, 0.0f);
      lw_s[i] = make_float4(u.x, u.y, w.x, w.y);
    }
  } else if (mel_in_smem) {
    for (int i = tid; i < a.mel_nnz; i += S::THREADS) melw_s[i] = __ldg(a.mel_pw + i);
  }
  const float *melw = mel_in_smem ? melw_s : a.mel_pw;
  __syncthreads();

  // W_64^j0: the odd half's extra rotation in the column combine
  const cpx w1 = j0 ? cpx{(float)ce_trig(1, 64, 0), -(float)ce_trig(1, 64, 1)} : cpx{1.0f, 0.0f};

  cpx *fb = bufs + fp * S::FSTRIDE;
  // power spectrum, padded: bin k at k + min(k / 32, 63), so that walk lane
  // j reads its bins [32 j, 32 j + 32) at 33 j + b and the Nyquist bin at 2111
  float *P = reinterpret_cast<float *>(fb);

  const int total = a.total_tiles;
  const int t_begin = (int)((long long)blockIdx.x * total / gridDim.x);
  const int t_end = (int)((long long)(blockIdx.x + 1) * total / gridDim.x);
  int cur = -1;
  float vmax = -INFINITY;

  for (int tile = t_begin; tile < t_end; tile++) {
    const int cl = __ldg(a.tile_clip + tile);
    if (cl != cur) {  // CTA-uniform: every frame of a tile belongs to one clip
      float m = vmax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
      if (lane == 0 && cur >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur, enc_f(m));
      cur = cl;
      vmax = -INFINITY;
    }
    const ClipDesc cd = load_clip(a.clips + cl);
    const int t = (tile - cd.tile_base) * F + fp;
    if (t >= cd.n_frames) continue;  // uniform over the warp pair
    const long long s0 = (long long)t * a.hop - a.pad;
    const float *sig = a.signal + cd.sig_off;

    // ---- gather: v[r] = (x[2n], x[2n+1]) for n = j + 64 r
    cpx v[32];
    if (s0 >= 0 && s0 + N <= cd.length) {
      const float *base = sig + s0 + 2 * j;
      if (((cd.sig_off + s0) & 1) == 0) {
#pragma unroll
        for (int r = 0; r < 32; r++) {
          const float2 x = __ldg(reinterpret_cast<const float2 *>(base + 2 * TPF * r));
          v[r] = {x.x, x.y};
        }
      } else {
#pragma unroll
        for (int r = 0; r < 32; r++) v[r] = {__ldg(base + 2 * TPF * r), __ldg(base + 2 * TPF * r + 1)};
      }
    } else {
      cpx tmp[32];
      gather_edge(tmp, sig, s0 + 2 * j, cd.length, a.pad_mode, 2 * TPF);
#pragma unroll
      for (int r = 0; r < 32; r++) v[r] = tmp[r];
    }
    // ---- window
    {
      const float4 *wb = win_s + j;
#pragma unroll
      for (int r = 0; r < 32; r += 2) {
        const float4 w = wb[TPF * (r / 2)];
        v[r].x *= w.x;
        v[r].y *= w.y;
        v[r + 1].x *= w.z;
        v[r + 1].y *= w.w;
      }
    }

    // ---- stage 1: 32-point DFT over registers, twiddle, row j of the buffer
    frame_sync<TPF>(fp);  // the previous frame's band reads of the buffer are done
    {
      cpx e[16], o[16];
#pragma unroll
      for (int m = 0; m < 16; m++) {
        e[m] = v[2 * m];
        o[m] = v[2 * m + 1];
      }
      dft16(e);
      dft16(o);
      cpx *row = fb + j * 33;
      const float4 t78 = tw4[7 * TPF + j];  // k = 15, 16
      const cpx g16 = {t78.z, t78.w};      // W_M^(16 j)
      float4 tp = t78;
      static_for<0, 16>([&](auto ki) {
        constexpr int k = decltype(ki)::value;
        const cpx tt = tw_const<k, 32>(o[k]);
        cpx lo = cadd(e[k], tt), hi = csub(e[k], tt);
        if constexpr (k > 0) {
          // pair k / 2 holds k (odd) and k + 1
          if constexpr (k == 15) tp = t78;
          else if constexpr (k % 2 == 1) tp = tw4[(k / 2) * TPF + j];
          const cpx tk = (k % 2 == 1) ? cpx{tp.x, tp.y} : cpx{tp.z, tp.w};
          lo = cmul(lo, tk);
          hi = cmul(hi, cmul(tk, g16));
        } else {
          hi = cmul(hi, g16);
        }
        row[k] = lo;
        row[k + 16] = hi;
      });
    }
    frame_sync<TPF>(fp);
    // ---- stage 2a: 32-point DFT of rows j0 + 2 j1 of column col -> A_j0[q]
#pragma unroll
    for (int j1 = 0; j1 < 32; j1++) v[j1] = fb[(j0 + 2 * j1) * 33 + col];
    dft32(v);
    // ---- stage 2b: combine the column's two halves; z[i] = Z[col + 32 (2i + j0)],
    // z[16 + i] = Z[col + 32 (2i + j0 + 32)]
    cpx z[32];
    static_for<0, 16>([&](auto ii) {
      constexpr int i = decltype(ii)::value;
      const cpx snd = j0 ? v[2 * i] : v[2 * i + 1];
      cpx rcv;
      rcv.x = __shfl_xor_sync(FULL, snd.x, 1);
      rcv.y = __shfl_xor_sync(FULL, snd.y, 1);
      const cpx ev = j0 ? rcv : v[2 * i];
      cpx od = tw_const<2 * i, 64>(j0 ? v[2 * i + 1] : rcv);
      od = cmul(od, w1);
      z[i] = cadd(ev, od);
      z[16 + i] = csub(ev, od);
    });
    // ---- real split: pair i is (Z[k], Z[M - k]), k = col + 32 (2i + j0); the
    // partner's z[31 - i] holds Z[M - k] (column 0: this thread's own z)
    cpx rcv[16];
#pragma unroll
    for (int m = 0; m < 16; m++) {
      rcv[m].x = __shfl_sync(FULL, z[16 + m].x, partner);
      rcv[m].y = __shfl_sync(FULL, z[16 + m].y, partner);
    }
    frame_sync<TPF>(fp);  // every column is read: the buffer becomes P
    {
      float *Pa = P + col + 33 * j0;                         // bin col + 32 s at col + 33 s
      float *Pb = P + (2111 - col - 33 * j0) + (c0 ? 1 : 0);  // bin M - col - 32 s
      float4 rsp;
      static_for<0, 16>([&](auto ii) {
        constexpr int i = decltype(ii)::value;
        const cpx za = z[i];
        cpx zb;
        if constexpr (i == 0) zb = c0 ? (j0 ? z[31] : z[0]) : rcv[15];
        else zb = c0 ? (j0 ? z[31 - i] : z[32 - i]) : rcv[15 - i];
        const float ex = za.x + zb.x, ey = za.y - zb.y;
        const float ox = za.y + zb.y, oy = zb.x - za.x;
        if constexpr (i % 2 == 0) rsp = rs_tw[(i + j0) * 33 + col];  // row 2 (i / 2) + j0
        const cpx w = (i % 2 == 0) ? cpx{rsp.x, rsp.y} : cpx{rsp.z, rsp.w};  // W_N^k
        const float wr = fmaf(w.x, ox, -w.y * oy), wi = fmaf(w.x, oy, w.y * ox);
        const float xr = ex + wr, xi = ey + wi;
        const float yr = ex - wr, yi = ey - wi;
        Pa[66 * i] = fmaf(xr, xr, xi * xi);
        const float q = fmaf(yr, yr, yi * yi);
        if constexpr (i == 0) Pb[(c0 && !j0) ? -1 : 0] = q;  // column 0, s = 0: the Nyquist bin
        else Pb[-66 * i] = q;
      });
      if (c0 && !j0) P[M / 2 + 32] = 4.0f * fmaf(z[16].x, z[16].x, z[16].y * z[16].y);
    }
    frame_sync<TPF>(fp);  // P complete

    // ---- log-mel row of this frame + running clip max
    float *dst = a.out + (cd.frame_off + t) * (long long)nmel;
    if (lanes) {
      // the filterbank walk of the single-warp kernel over 64 lanes (and its
      // non-finite check: p * 0 accumulated over the bins)
      float2 *parts = reinterpret_cast<float2 *>(P + 33 * TPF);
      const int2 li = lane_s[j];
      const unsigned fl = (unsigned)li.x;
      int slot = li.y & 1023;
      const float *pl = P + 33 * j;
      const float4 *wl = lw_s + j;
      float R = 0.0f, Fs = 0.0f, tot = 0.0f;
      float4 wq;
#pragma unroll
      for (int b = 0; b < 32; b++) {
        const float p = pl[b];
        if ((b & 1) == 0) wq = wl[(b >> 1) * TPF];
        const float2 w = (b & 1) ? make_float2(wq.z, wq.w) : make_float2(wq.x, wq.y);
        tot = fmaf(p, 0.0f, tot);
        R = fmaf(w.x, p, R);
        Fs = fmaf(w.y, p, Fs);
        if (fl & (1u << b)) {
          parts[slot++] = make_float2(R, Fs);
          R = 0.0f;
          Fs = 0.0f;
        }
      }
      if (j == TPF - 1) {
        const float p = pl[32];
        const float4 wn = wl[16 * TPF];
        const float2 w = make_float2(wn.x, wn.y);
        tot = fmaf(p, 0.0f, tot);
        R = fmaf(w.x, p, R);
        Fs = fmaf(w.y, p, Fs);
        parts[slot] = make_float2(R, Fs);
      }
      if (j == 0) parts[li.y >> 16] = make_float2(0.0f, 0.0f);  // the empty segments' slot
      const bool bad = frame_sync_or<TPF>(fp, !isfinite(tot));
      const int kc = (li.y >> 10) & 63;
      if (kc) {
        const int h = j == TPF - 1 ? slot : slot - 1;
        float2 hv = parts[h];
        for (int q = 1; q <= kc; q++) {
          const float2 pv = parts[h + q];
          hv.x += pv.x;
          hv.y += pv.y;
        }
        parts[h] = hv;
      }
      frame_sync<TPF>(fp);
      for (int m = j; m < nmel; m += TPF) {
        const int bw = band_s[m];
        float acc = parts[bw & 4095].x + parts[(bw >> 12) & 4095].y;
        if (((bw >> 24) & 1) || bad) acc = __int_as_float(0x7fc00000);
        const float val = db10_frame(acc, a.amin, ref_db);
        dst[m] = val;
        vmax = fmaxf(vmax, val);
      }
    } else {
      float chk = 0.0f;  // the frame's non-finite check: this thread's share of the bins, times 0
      for (int k = j; k <= M; k += TPF) chk = fmaf(P[pad_bin<TPF>(k)], 0.0f, chk);
      const bool bad = frame_sync_or<TPF>(fp, !isfinite(chk));
      for (int m = j; m < nmel; m += TPF) {
        const float acc = mel_dot_pad<TPF>(__ldg(a.mel_info + m), melw, P, bad);
        const float val = db10_frame(acc, a.amin, ref_db);
        dst[m] = val;
        vmax = fmaxf(vmax, val);
      }
    }
  }
  float m = vmax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
  if (lane == 0 && cur >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur, enc_f(m));
}

// ---------------------------------------------------------------------------
// n_fft 2048 with both 32-point DFT stages on the tensor cores (launch
// variant 5).  The frame is the packed sequence z[n] (n = n1 + 32 n2) of the
// warp kernel, 1 024 complex points as 32 x 32:
//
//   stage 1  Y[n1][k2] = sum_n2 z[n1 + 32 n2] W_32^(n2 k2)      (GEMM 1)
//   twiddle  Y[n1][k2] *= W_1024^(n1 k2)                         (CUDA cores)
//   stage 2  Z[k2 + 32 k1] = sum_n1 Y[n1][k2] W_32^(n1 k1)      (GEMM 2)
//
// Both GEMMs take the same B: the 32-point DFT in real form (64 x 64, inputs
// [re | im], outputs [re | im]), built in float64 and split into fp16 hi +
// lo parts.  Four frames make one M = 128 tile: GEMM 1's A has a row per
// (frame, n1) and K = [re z | im z] over n2 (K-major, the lane of a warp
// holds its row); GEMM 2's A has a row per (frame, k2) and K over n1, and is
// written MN-major (lane n1 holds K-rows n1 and 32 + n1, each 32 contiguous
// values along M).  Each GEMM is hi*hi + hi*lo + lo*hi in fp16 with float32
// accumulation in tensor memory, 12 tcgen05.mma of M 128 x N 64 x K 16,
// issued by one thread.  fp16 needs the frame in range: the windowed samples
// are scaled by 2^-e (their largest magnitude into [0.5, 1)), which keeps the
// split at float32 grade (the lo parts of small values keep 2^-24 of the
// frame's largest sample), and the band sums are scaled back by 2^(2e),
// exactly.  GEMM 2's output row (frame, k2) holds Z[k2 + 32 k1] for all k1,
// the register layout of the warp kernel after its stage 2, so the real
// split, the filterbank walk, the log and the running clip maximum are the
// warp kernel's.
//
// CTA: 16 warps in 4 independent groups of 4 (one frame per warp, one M = 128
// tile per group), one CTA per SM holding 256 tensor-memory columns (64 per
// group).  A group's shared region holds its A images (hi, lo; reused by
// both GEMMs) and, after GEMM 2 has completed, the four frames' spectra.  Per
// tile a group synchronises on three named barriers (A1 written, A2 written,
// spectra read) and two mbarriers the MMA commits arrive on.  Every mbarrier
// wait is bounded: a wait that runs out sets *a.err, the group leaves the
// loop together at its next barrier (a barrier reduction), and the CTA waits
// (bounded) for its MMAs before releasing tensor memory.
// ---------------------------------------------------------------------------
struct TcShape {
  static constexpr int N = 2048, M = 1024, TPF = 32;
  static constexpr int NW = 16, THREADS = 512, GROUPS = 4, F = 16;  // frames per CTA tile
  static constexpr uint32_t IMG = 128 * 128;      // one A image: 128 rows x 64 fp16 (16 KB)
  static constexpr uint32_t FBUF = 33 * 32 * 8;   // one frame's padded spectrum + part slots (bytes)
  static constexpr uint32_t REGION = 34 * 1024;   // per group: A hi + lo, later 4 spectra (1024-aligned)
  static constexpr uint32_t BIMG = 64 * 128;      // one B image: 64 rows x 64 fp16 (8 KB)
  static constexpr int MEL_SMEM_MAX = 8192;       // packed weights staged up to this many floats
};
static_assert(4 * TcShape::FBUF <= TcShape::REGION && 2 * TcShape::IMG <= TcShape::REGION, "group region");

struct TcSmem {
  uint32_t region, b, tw2, win, rs, mel, bar, taddr, total;
};
__host__ __device__ inline TcSmem tc_smem_layout(int n_mels, bool lanes, int nnz) {
  using S = TcShape;
  TcSmem L{};
  uint32_t p = 0;
  L.region = p;
  p += S::GROUPS * S::REGION;
  L.b = p;
  p += 2 * S::BIMG;
  L.tw2 = p;
  p += 31 * S::TPF * 8;
  L.win = p;
  p += S::N * 4;
  L.rs = p;
  p += 16 * 32 * 8;
  L.mel = p;
  if (lanes)
    p += (uint32_t)(align16(4 * (size_t)n_mels) + 8 * S::TPF + 33 * S::TPF * 8);
  else
    p += (uint32_t)(16 * (size_t)n_mels + (nnz <= S::MEL_SMEM_MAX ? align16(4 * (size_t)nnz) : 0));
  p = (p + 15u) & ~15u;
  L.bar = p;  // per group: GEMM 1 done, GEMM 2 done; then the exit barrier
  p += 8 * (2 * S::GROUPS + 1);
  p = (p + 15u) & ~15u;
  L.taddr = p;
  p += 16;
  L.total = p + 1024;  // slack to align the base to 1024 bytes
  return L;
}

// Named barrier over the 128 threads of group g (ids 1..4), returning whether
// any of them passed `pred`.
__device__ __forceinline__ bool group_sync_or(int g, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(g + 1)
      : "memory");
  return r != 0;
}

// Two fp16 parts of 8 floats (|x| < 1), packed for one 16-byte store each.
// The hi part is x rounded to 11 significant bits in the float32 domain
// (integer add and mask on the bits), so lo = x - hi is exact in float32 and
// no fp16 value is converted back: only the two packing conversions remain.
// (hi converts to fp16 exactly unless it falls below fp16's normal range,
// where the error is at most 2^-25, far below the frame's largest sample.)
__device__ __forceinline__ void split8_half(const float *x, uint4 &hi, uint4 &lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float h0 = __uint_as_float((__float_as_uint(x[2 * i]) + 0x1000u) & 0xFFFFE000u);
    const float h1 = __uint_as_float((__float_as_uint(x[2 * i + 1]) + 0x1000u) & 0xFFFFE000u);
    const __half2 a = __floats2half2_rn(h0, h1);
    const __half2 b = __floats2half2_rn(x[2 * i] - h0, x[2 * i + 1] - h1);
    h[i] = *reinterpret_cast<const uint32_t *>(&a);
    l[i] = *reinterpret_cast<const uint32_t *>(&b);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(TcShape::THREADS, 1) frame_tc_kernel(FrontArgs a) {
  using S = TcShape;
  constexpr int N = S::N, M = S::M, TPF = S::TPF;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char tc_raw[];
  const uint32_t raw = smem_u32(tc_raw);
  unsigned char *sm = tc_raw + (((raw + 1023u) & ~1023u) - raw);
  const int nmel = a.n_mels;
  const bool lanes = a.mel_lane_ok != 0;
  const bool mel_in_smem = a.mel_nnz <= S::MEL_SMEM_MAX;
  const TcSmem Ly = tc_smem_layout(nmel, lanes, a.mel_nnz);
  cpx *tw2 = reinterpret_cast<cpx *>(sm + Ly.tw2);      // W_M^(j k1), [k1-1][j]
  float *win_s = reinterpret_cast<float *>(sm + Ly.win);  // analysis window, halved
  cpx *rs_tw = reinterpret_cast<cpx *>(sm + Ly.rs);     // real-split twiddles [32 i + l]
  unsigned char *mp = sm + Ly.mel;
  int *band_s = reinterpret_cast<int *>(mp);
  int2 *lane_s = reinterpret_cast<int2 *>(mp + align16(4 * (size_t)nmel));
  float2 *lw_s = reinterpret_cast<float2 *>(mp + align16(4 * (size_t)nmel) + 8 * TPF);
  int4 *mel_s = reinterpret_cast<int4 *>(mp);
  float *melw_s = reinterpret_cast<float *>(mp + 16 * (size_t)nmel);
  const uint32_t bar0 = smem_u32(sm + Ly.bar);
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(sm + Ly.taddr);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = warp >> 2, w4 = warp & 3;  // MMA group, frame within the group
  const float2 *twq = a.tw_split;
  unsigned char *region = sm + Ly.region + g * S::REGION;
  const uint32_t a_hi = smem_u32(region), a_lo = a_hi + S::IMG;
  const uint32_t b_hi = smem_u32(sm + Ly.b), b_lo = b_hi + S::BIMG;
  const uint32_t bar_g1 = bar0 + 16u * (uint32_t)g, bar_g2 = bar_g1 + 8u, bar_fin = bar0 + 16u * S::GROUPS;

  // ---- tables: the real-form 32-point DFT as fp16 hi/lo images (float64),
  // B[n][k] for output n = 32 c_out + k' and input k = 32 c_in + n'
  for (int i = tid; i < 64 * 64; i += S::THREADS) {
    const int n = i >> 6, k = i & 63;
    const int co = n >> 5, ci = k >> 5;
    double sn, cs;
    sincospi(2.0 * (double)(((n & 31) * (k & 31)) & 31) / 32.0, &sn, &cs);
    const double v = (co == ci) ? cs : (co == 0 ? sn : -sn);
    const __half hi = __double2half(v);
    const __half lo = __double2half(v - (double)__half2float(hi));
    *reinterpret_cast<__half *>(sm + Ly.b + sw128(n, k)) = hi;
    *reinterpret_cast<__half *>(sm + Ly.b + S::BIMG + sw128(n, k)) = lo;
  }
  for (int i = tid; i < 31 * TPF; i += S::THREADS) {
    const int k1 = i / TPF + 1, j = i - (k1 - 1) * TPF;
    tw2[i] = root_q(twq, 2 * j * k1, N);
  }
  for (int i = tid; i < N / 4; i += S::THREADS) {  // halved: see the warp kernel
    const float4 w = __ldg(reinterpret_cast<const float4 *>(a.window) + i);
    reinterpret_cast<float4 *>(win_s)[i] = make_float4(0.5f * w.x, 0.5f * w.y, 0.5f * w.z, 0.5f * w.w);
  }
  for (int i = tid; i < 16 * 32; i += S::THREADS) rs_tw[i] = root_q(twq, (i & 31) + 32 * (i >> 5), N);
  if (lanes) {
    for (int i = tid; i < nmel; i += S::THREADS) band_s[i] = __ldg(a.mel_band + i);
    for (int i = tid; i < TPF; i += S::THREADS) lane_s[i] = __ldg(a.mel_lane + i);
    for (int i = tid; i < 33 * TPF; i += S::THREADS) lw_s[i] = __ldg(a.mel_lw + i);
  } else {
    for (int i = tid; i < nmel; i += S::THREADS) mel_s[i] = __ldg(a.mel_info + i);
    if (mel_in_smem)
      for (int i = tid; i < a.mel_nnz; i += S::THREADS) melw_s[i] = __ldg(a.mel_pw + i);
  }
  const float *melw = mel_in_smem ? melw_s : a.mel_pw;
  if (tid == 0) {
    for (int q = 0; q < 2 * S::GROUPS; q++) mbar_init(bar0 + 8u * q, 1);
    mbar_init(bar0 + 8u * (2 * S::GROUPS), S::GROUPS);  // one final commit per group
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();  // the B images are read by the tensor core
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;
  const uint32_t acc = tmem + (uint32_t)(64 * g);               // this group's 64 columns
  const uint32_t tl = acc + ((uint32_t)(32 * w4) << 16);         // this warp's lane quarter
  constexpr uint32_t kId1 = idesc_f16kind<true>(64, 128, false);  // A K-major
  constexpr uint32_t kId2 = idesc_f16kind<true>(64, 128, true);   // A MN-major
  const bool issuer = (w4 == 0) && (lane == 0);

  float *P = reinterpret_cast<float *>(region + w4 * S::FBUF);
  const float ref_db = 10.0f * log10f(a.ref);
  const int total = a.total_tiles;
  const int t_begin = (int)((long long)blockIdx.x * total / gridDim.x);
  const int t_end = (int)((long long)(blockIdx.x + 1) * total / gridDim.x);
  int cur = -1;
  float vmax = -INFINITY;
  uint32_t it = 0;
  bool failed = false;

  for (int tile = t_begin; tile < t_end; tile++, it++) {
    const int c = __ldg(a.tile_clip + tile);
    if (c != cur) {  // warp-uniform: every frame of a tile belongs to one clip
      float m = vmax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
      if (lane == 0 && cur >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur, enc_f(m));
      cur = c;
      vmax = -INFINITY;
    }
    const ClipDesc cd = load_clip(a.clips + c);
    const int t = (tile - cd.tile_base) * S::F + 4 * g + w4;
    const bool valid = t < cd.n_frames;  // warp-uniform; a frame past the clip computes zeros
    const long long s0 = (long long)t * a.hop - a.pad;
    const float *sig = a.signal + cd.sig_off;

    // ---- gather + window: v[r] = (x[2n], x[2n+1]) w / 2 for n = lane + 32 r
    cpx v[32];
    if (!valid) {
#pragma unroll
      for (int r = 0; r < 32; r++) v[r] = {0.0f, 0.0f};
    } else if (s0 >= 0 && s0 + N <= cd.length) {
      const float *base = sig + s0 + 2 * lane;
      if (((cd.sig_off + s0) & 1) == 0) {
#pragma unroll
        for (int r = 0; r < 32; r++) {
          const float2 x = __ldg(reinterpret_cast<const float2 *>(base + 2 * TPF * r));
          v[r] = {x.x, x.y};
        }
      } else {
#pragma unroll
        for (int r = 0; r < 32; r++) v[r] = {__ldg(base + 2 * TPF * r), __ldg(base + 2 * TPF * r + 1)};
      }
    } else {
      cpx tmp[32];
      gather_edge(tmp, sig, s0 + 2 * lane, cd.length, a.pad_mode, 2 * TPF);
#pragma unroll
      for (int r = 0; r < 32; r++) v[r] = tmp[r];
    }
    float mx = 0.0f;
    {
      const float2 *wb = reinterpret_cast<const float2 *>(win_s) + lane;
#pragma unroll
      for (int r = 0; r < 32; r++) {
        const float2 w = wb[TPF * r];
        v[r].x *= w.x;
        v[r].y *= w.y;
        mx = fmaxf(mx, fmaxf(fabsf(v[r].x), fabsf(v[r].y)));  // NaNs are ignored here
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
    // 2^-e with the frame's largest windowed sample in [0.5, 1); 1 for a frame
    // of zeros or one with an infinite sample
    int e = 0;
    if (mx > 0.0f && mx <= 3.402823466e38f) e = min(60, max(-60, ilogbf(mx) + 1));
    const float sc = __int_as_float((127 - e) << 23);
    const float isc2 = __int_as_float((127 + 2 * e) << 23);

    // ---- GEMM 1's A: row 32 w4 + lane, K = [re z | im z] over n2 (K-major)
    {
      const int row = 32 * w4 + lane;
#pragma unroll
      for (int c8 = 0; c8 < 8; c8++) {
        float xs[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const cpx z = v[(c8 & 3) * 8 + u];
          xs[u] = (c8 < 4 ? z.x : z.y) * sc;
        }
        uint4 hi, lo;
        split8_half(xs, hi, lo);
        const uint32_t off = sw128(row, 8 * c8);
        *reinterpret_cast<uint4 *>(region + off) = hi;
        *reinterpret_cast<uint4 *>(region + S::IMG + off) = lo;
      }
    }
    fence_proxy_async_smem();
    group_sync_or(g, false);
    if (issuer) {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint64_t ah = desc_sw128(a_hi + 32u * k), al = desc_sw128(a_lo + 32u * k);
        const uint64_t bh = desc_sw128(b_hi + 32u * k), bl = desc_sw128(b_lo + 32u * k);
        umma_f16kind(acc, ah, bh, kId1, k > 0 ? 1u : 0u);
        umma_f16kind(acc, ah, bl, kId1, 1u);
        umma_f16kind(acc, al, bh, kId1, 1u);
      }
      umma_commit(bar_g1);
    }
    bool ok = mbar_wait_bounded(bar_g1, it & 1u);
    tc_fence_after();

    // ---- GEMM 1's result: lane n1 holds Y[n1][k2] (columns k2 and 32 + k2)
    float y[64];  // [re | im]
    if (ok) {
      tmem_ld64(tl, y);
    } else {
#pragma unroll
      for (int q = 0; q < 64; q++) y[q] = 0.0f;
    }
    float *yr = y, *yi = y + 32;
    // twiddle W_M^(n1 k2)
#pragma unroll
    for (int k2 = 1; k2 < 32; k2++) {
      const cpx r = cmul(cpx{yr[k2], yi[k2]}, tw2[(k2 - 1) * TPF + lane]);
      yr[k2] = r.x;
      yi[k2] = r.y;
    }
    // ---- GEMM 2's A (MN-major): K-rows n1 (re) and 32 + n1 (im), M = 32 w4 + k2;
    // atoms of 64 M x 8 K-rows, 1024 bytes apart along M, 2048 along K
    {
      const uint32_t iblk = (uint32_t)(w4 >> 1) * 1024u;
      const int cm0 = 4 * (w4 & 1);
#pragma unroll
      for (int part = 0; part < 2; part++) {
        const int kidx = part * 32 + lane;
        const uint32_t kbase = (uint32_t)(kidx >> 3) * 2048u + iblk + (uint32_t)(kidx & 7) * 128u;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          uint4 hi, lo;
          split8_half(part ? yi + 8 * q : yr + 8 * q, hi, lo);
          const uint32_t off = kbase + ((uint32_t)((cm0 + q) ^ (kidx & 7)) << 4);
          *reinterpret_cast<uint4 *>(region + off) = hi;
          *reinterpret_cast<uint4 *>(region + S::IMG + off) = lo;
        }
      }
    }
    tc_fence_before();  // this warp's tensor-memory loads are complete (tcgen05.wait::ld)
    fence_proxy_async_smem();
    if (group_sync_or(g, !ok)) {
      failed = true;
      break;
    }
    if (issuer) {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint64_t ah = desc_mn_sw128(a_hi + 4096u * k, 1024u, 2048u);
        const uint64_t al = desc_mn_sw128(a_lo + 4096u * k, 1024u, 2048u);
        const uint64_t bh = desc_sw128(b_hi + 32u * k), bl = desc_sw128(b_lo + 32u * k);
        umma_f16kind(acc, ah, bh, kId2, k > 0 ? 1u : 0u);
        umma_f16kind(acc, ah, bl, kId2, 1u);
        umma_f16kind(acc, al, bh, kId2, 1u);
      }
      umma_commit(bar_g2);
    }
    ok = mbar_wait_bounded(bar_g2, it & 1u);
    tc_fence_after();
    // ---- GEMM 2's result: lane l = k2 of this frame holds v[k1] = Z[l + 32 k1]
    if (ok) tmem_ld64(tl, y);
#pragma unroll
    for (int k1 = 0; k1 < 32; k1++) v[k1] = {y[k1], y[32 + k1]};
    tc_fence_before();
    // the spectra alias the A images: every MMA of the group has completed
    // (each warp waited on GEMM 2's barrier), and no warp writes A before the
    // barrier at the end of this tile

    // ---- real split, P[k] = |X[k] sc|^2 (the window was halved), as the warp kernel (C == 1)
    {
      const int l = lane;
      const int src = (32 - l) & 31;
      cpx rcv[16];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        rcv[q].x = __shfl_sync(FULL, v[16 + q].x, src);
        rcv[q].y = __shfl_sync(FULL, v[16 + q].y, src);
      }
      const bool l0 = (l == 0);
      float *Pa = P + l;
      float *Pb = P + (M + TPF - 1 - l) + (l0 ? 1 : 0);
      static_for<0, 16>([&](auto ki) {
        constexpr int i = decltype(ki)::value;
        const cpx za = v[i];
        cpx zb;
        if constexpr (i == 0) zb = l0 ? v[0] : rcv[15];
        else zb = l0 ? rcv[16 - i] : rcv[15 - i];
        const float ex = za.x + zb.x, ey = za.y - zb.y;
        const float ox = za.y + zb.y, oy = zb.x - za.x;
        const cpx w = rs_tw[32 * i + l];
        const float wr = fmaf(w.x, ox, -w.y * oy), wi = fmaf(w.x, oy, w.y * ox);
        const float xr = ex + wr, xi = ey + wi;
        const float yr2 = ex - wr, yi2 = ey - wi;
        const float p = fmaf(xr, xr, xi * xi), q = fmaf(yr2, yr2, yi2 * yi2);
        Pa[33 * i] = p;
        if constexpr (i == 0) Pb[l0 ? -1 : 0] = q;
        else Pb[-33 * i] = q;
      });
      if (l0) P[M / 2 + TPF / 2] = 4.0f * fmaf(rcv[0].x, rcv[0].x, rcv[0].y * rcv[0].y);
    }
    __syncwarp();  // P complete

    // ---- log-mel row + running clip max: band sums scaled back by 2^(2e)
    float *dst = a.out + (cd.frame_off + t) * (long long)nmel;
    const bool out = valid && ok;  // (a failed wait: the group stops at the barrier below)
    if (lanes) {
      float2 *parts = reinterpret_cast<float2 *>(P + 33 * TPF);
      const int l = lane;
      const int2 li = lane_s[l];
      const unsigned fl = (unsigned)li.x;
      int slot = li.y & 1023;
      const float *pl = P + 33 * l;
      const float2 *wl = lw_s + l;
      float R = 0.0f, Fs = 0.0f, tot = 0.0f;
#pragma unroll
      for (int b = 0; b < 32; b++) {
        const float p = pl[b];
        const float2 w = wl[b * TPF];
        tot = fmaf(p, 0.0f, tot);
        R = fmaf(w.x, p, R);
        Fs = fmaf(w.y, p, Fs);
        if (fl & (1u << b)) {
          parts[slot++] = make_float2(R, Fs);
          R = 0.0f;
          Fs = 0.0f;
        }
      }
      if (l == TPF - 1) {
        const float p = pl[32];
        const float2 w = wl[32 * TPF];
        tot = fmaf(p, 0.0f, tot);
        R = fmaf(w.x, p, R);
        Fs = fmaf(w.y, p, Fs);
        parts[slot] = make_float2(R, Fs);
      }
      if (e > 53) {  // |X|^2 itself may overflow float32 only for samples this large
        float pm = 0.0f;
        for (int b = 0; b <= (l == TPF - 1 ? 32 : 31); b++) pm = fmaxf(pm, pl[b]);
        tot = fmaf(pm * isc2, 0.0f, tot);
      }
      const bool bad = __ballot_sync(FULL, !isfinite(tot)) != 0;
      if (l == 0) parts[li.y >> 16] = make_float2(0.0f, 0.0f);
      __syncwarp();
      const int kc = (li.y >> 10) & 63;
      if (kc) {
        const int h = l == TPF - 1 ? slot : slot - 1;
        float2 hv = parts[h];
        for (int j = 1; j <= kc; j++) {
          const float2 pv = parts[h + j];
          hv.x += pv.x;
          hv.y += pv.y;
        }
        parts[h] = hv;
      }
      __syncwarp();
      for (int m = l; m < nmel; m += TPF) {
        const int bw = band_s[m];
        float accm = (parts[bw & 4095].x + parts[(bw >> 12) & 4095].y) * isc2;
        if (((bw >> 24) & 1) || bad) accm = __int_as_float(0x7fc00000);
        const float val = db10_frame(accm, a.amin, ref_db);
        if (out) {
          dst[m] = val;
          vmax = fmaxf(vmax, val);
        }
      }
    } else {
      float chk = 0.0f;
      float pm = 0.0f;
      for (int k = lane; k <= M; k += TPF) {
        const float p = P[pad_bin<TPF>(k)];
        chk = fmaf(p, 0.0f, chk);
        pm = fmaxf(pm, p);
      }
      if (e > 53) chk = fmaf(pm * isc2, 0.0f, chk);
      const bool bad = __ballot_sync(FULL, !isfinite(chk)) != 0;
      for (int m = lane; m < nmel; m += TPF) {
        const float accm = mel_dot_pad<TPF>(mel_s[m], melw, P, bad) * isc2;
        const float val = db10_frame(accm, a.amin, ref_db);
        if (out) {
          dst[m] = val;
          vmax = fmaxf(vmax, val);
        }
      }
    }
    // the spectra are read before the next tile's A overwrites them; a failed
    // GEMM 2 wait ends the loop for the whole group here
    if (group_sync_or(g, !ok)) {
      failed = true;
      break;
    }
  }
  if (failed && lane == 0) atomicOr(a.err, 1u);
  float m = vmax;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
  if (!failed && lane == 0 && cur >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur, enc_f(m));
  // every MMA this group issued has completed before tensor memory is released
  if (issuer) {
    umma_commit(bar_fin);  // arrives once the group's MMAs are done (one arrival per group issuer)
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0) mbar_wait_bounded(bar_fin, 0u);
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

cudaError_t launch_frontend_tc(const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched) {
  using S = TcShape;
  if (launched) *launched = 0;
  if (a.total_tiles <= 0) return cudaSuccess;
  if (!a.err) return cudaErrorInvalidValue;  // bounded waits report through the error word
  const size_t smem = tc_smem_layout(a.n_mels, a.mel_lane_ok != 0, a.mel_nnz).total;
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  int per_sm = 1, sms = 148;
  cudaError_t e =
      persistent_geometry(reinterpret_cast<const void *>(frame_tc_kernel), S::THREADS, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = sms;  // one CTA per SM: 256 of the SM's 512 tensor-memory columns
  if (grid_limit > 0 && grid > grid_limit) grid = grid_limit;
  if (grid > a.total_tiles) grid = a.total_tiles;
  frame_tc_kernel<<<(unsigned)grid, S::THREADS, smem, s>>>(a);
  if (launched) *launched = (int)grid;
  return cudaGetLastError();
}

static cudaError_t launch_warp2(const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched) {
  using S = W2Shape;
  // lane walk: band words, lane words (8 TPF), weight pairs (17 x TPF float4)
  const size_t tables = a.mel_lane_ok ? align16(4 * (size_t)a.n_mels) + 8 * (size_t)S::TPF + 16 * 17 * (size_t)S::TPF
                                      : (a.mel_nnz <= S::MEL_SMEM_MAX ? align16(4 * (size_t)a.mel_nnz) : 0);
  const size_t smem = warp2_fixed_smem() + tables;
  int per_sm = 1, sms = 148;
  cudaError_t e =
      persistent_geometry(reinterpret_cast<const void *>(frame_warp2_kernel), S::THREADS, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = (long long)sms * per_sm;
  if (grid_limit > 0 && grid > grid_limit) grid = grid_limit;
  if (grid > a.total_tiles) grid = a.total_tiles;
  if (grid < 1) return cudaSuccess;
  frame_warp2_kernel<<<(unsigned)grid, S::THREADS, smem, s>>>(a);
  if (launched) *launched = (int)grid;
  return cudaGetLastError();
}

template <int LOG2N>
static cudaError_t launch_warp_t(const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched) {
  using S = WShape<LOG2N>;
  // lane walk: band words (4 n_mels, 16-aligned), lane words (8 TPF), weight
  // pairs (17 x TPF float4); else the packed rows
  const size_t tables = a.mel_lane_ok ? align16(4 * (size_t)a.n_mels) + 8 * (size_t)S::TPF + 16 * 17 * (size_t)S::TPF
                                      : mel_smem_bytes(a.n_mels, a.mel_nnz);
  const size_t smem = warp_fixed_smem<LOG2N>() + tables;
  auto kern = frame_warp_kernel<LOG2N>;
  int per_sm = 1, sms = 148;
  cudaError_t e = persistent_geometry(reinterpret_cast<const void *>(kern), S::THREADS, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = (long long)sms * per_sm;
  if (grid_limit > 0 && grid > grid_limit) grid = grid_limit;
  if (grid > a.total_tiles) grid = a.total_tiles;
  if (grid < 1) return cudaSuccess;
  kern<<<(unsigned)grid, S::THREADS, smem, s>>>(a);
  if (launched) *launched = (int)grid;
  return cudaGetLastError();
}

cudaError_t launch_frontend_warp(int log2n, const FrontArgs &a, int grid_limit, cudaStream_t s,
                                 int *launched) {
  if (launched) *launched = 0;
  if (a.total_tiles <= 0) return cudaSuccess;
  switch (log2n) {
    case 8: return launch_warp_t<8>(a, grid_limit, s, launched);
    case 9: return launch_warp_t<9>(a, grid_limit, s, launched);
    case 10: return launch_warp_t<10>(a, grid_limit, s, launched);
    case 11: return launch_warp_t<11>(a, grid_limit, s, launched);
    case 12: return launch_warp2(a, grid_limit, s, launched);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mm
