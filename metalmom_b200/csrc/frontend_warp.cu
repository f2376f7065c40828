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
//   one shared-memory transpose (row stride 33, conflict-free)
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

#include "fft_radix.cuh"
#include "frame_common.cuh"
#include "kernels.h"

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
  static constexpr int FSTRIDE = TPF * 33;  // complex slots per frame buffer
  static constexpr int NW = 8;              // warps per CTA
  static constexpr int THREADS = 32 * NW;
  static constexpr int F = NW * FPW;        // frames per CTA tile
  static_assert(TPF >= 4 && TPF <= 32, "n_fft must be 256..2048");
};

// Real-split twiddles W_N^(l + 32 i), i < 16, of lane l (one frame per warp
// only): 512 complex, read as [32 i + l].
template <int LOG2N>
__host__ __device__ constexpr size_t warp_split_tw() {
  return WShape<LOG2N>::C == 1 ? size_t(16 * 32) * 8 : 0;
}

template <int LOG2N>
__host__ __device__ constexpr size_t warp_fixed_smem() {
  using S = WShape<LOG2N>;
  return align16(size_t(31) * S::TPF * 8) + align16(size_t(S::N) * 4) + warp_split_tw<LOG2N>() +
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

// Position of bin k in the padded power spectrum (k + min(k / 32, TPF - 1)).
template <int TPF>
__device__ __forceinline__ int pad_bin(int k) {
  const int q = k >> 5;
  return k + (q < TPF - 1 ? q : TPF - 1);
}

// mel_dot over the padded power spectrum.
template <int TPF>
__device__ __forceinline__ float mel_dot_pad(int4 info, const float *w, const float *P, bool bad) {
  const float *wr = w + info.z;
  float acc = 0.0f;
  for (int q = 0; q < info.y; q++) acc = fmaf(wr[q], P[pad_bin<TPF>(info.x + q)], acc);
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
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nmel = a.n_mels;
  const float ref_db = 10.0f * log10f(a.ref);
  // Lane walk over the per-bin split of the filterbank (else packed rows).
  const bool lanes = a.mel_lane_ok != 0;
  const bool mel_in_smem = a.mel_nnz <= kMelSmemMax;
  unsigned char *sp = smem;
  cpx *tw2 = reinterpret_cast<cpx *>(sp);  // W_M^(j k1), [k1-1][j]
  sp += align16(size_t(31) * TPF * 8);
  float *win_s = reinterpret_cast<float *>(sp);  // analysis window, natural order
  sp += align16(size_t(N) * 4);
  cpx *rs_tw = reinterpret_cast<cpx *>(sp);  // C == 1: real-split twiddles [32 i + l]
  sp += warp_split_tw<LOG2N>();
  cpx *bufs = reinterpret_cast<cpx *>(sp);
  sp += size_t(F) * S::FSTRIDE * 8;
  // lanes: band words, lane words, lane-minor weights; else packed rows
  int *band_s = reinterpret_cast<int *>(sp);
  int2 *lane_s = reinterpret_cast<int2 *>(sp + align16(4 * (size_t)nmel));
  float2 *lw_s = reinterpret_cast<float2 *>(sp + align16(4 * (size_t)nmel) + 8 * TPF);
  int4 *mel_s = reinterpret_cast<int4 *>(sp);
  float *melw_s = reinterpret_cast<float *>(sp + 16 * (size_t)nmel);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = lane / TPF;       // frame of this lane within the warp
  const int l = lane - grp * TPF;   // lane within the frame group
  const float2 *twq = a.tw_split;   // W_N^t, t < N/4

  for (int i = tid; i < 31 * TPF; i += S::THREADS) {
    const int k1 = i / TPF + 1, j = i - (k1 - 1) * TPF;
    tw2[i] = root_q(twq, 2 * j * k1, N);
  }
  for (int i = tid; i < N / 4; i += S::THREADS) {  // halved: see the header comment
    const float4 w = __ldg(reinterpret_cast<const float4 *>(a.window) + i);
    reinterpret_cast<float4 *>(win_s)[i] = make_float4(0.5f * w.x, 0.5f * w.y, 0.5f * w.z, 0.5f * w.w);
  }
  if constexpr (C == 1)
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
  // power spectrum, padded: bin k at k + min(k / 32, TPF - 1), so that lane l
  // of the group reads its bins [32 l, 32 l + 32) at 33 l + b, and the
  // Nyquist bin M at 33 TPF - 1; group g starts TPF g floats into its buffer
  // so that the groups of a warp fall in disjoint banks
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
      const float2 *wb = reinterpret_cast<const float2 *>(win_s) + l;
#pragma unroll
      for (int r = 0; r < 32; r++) {
        const float2 w = wb[TPF * r];
        v[r].x *= w.x;
        v[r].y *= w.y;
      }
    }

    // ---- stage 1: 32-point DFT over registers; its last butterflies are
    // followed directly by the twiddle W_M^(l k1) and the store into row l of
    // the frame buffer (stride 33), so that registers free up as it goes.
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
      const cpx g16 = tw2[15 * TPF + l];
      static_for<0, 16>([&](auto ki) {
        constexpr int k = decltype(ki)::value;
        const cpx t = tw_const<k, 32>(o[k]);
        cpx lo = cadd(e[k], t), hi = csub(e[k], t);
        if constexpr (k > 0) {
          const cpx tk = tw2[(k - 1) * TPF + l];
          lo = cmul(lo, tk);
          hi = cmul(hi, cmul(tk, g16));
        } else {
          hi = cmul(hi, g16);
        }
        row[k] = lo;
        row[k + 16] = hi;
      });
    }
    __syncwarp();
    static_for<0, C>([&](auto ci) {
      constexpr int cc = decltype(ci)::value;
      const int col = stage2_col<TPF, C, cc>(l);
#pragma unroll
      for (int jj = 0; jj < TPF; jj++) v[cc * TPF + jj] = fb[jj * 33 + col];
    });
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
      float *Pa = P + l;                              // bin l + 32 i at l + 33 i
      float *Pb = P + (M + TPF - 1 - l) + (l0 ? 1 : 0);  // bin M - l - 32 i, i > 0
      static_for<0, 16>([&](auto ki) {
        constexpr int i = decltype(ki)::value;
        const cpx za = v[i];
        cpx zb;
        if constexpr (i == 0) zb = l0 ? v[0] : rcv[15];
        else zb = l0 ? rcv[16 - i] : rcv[15 - i];
        const float ex = za.x + zb.x, ey = za.y - zb.y;
        const float ox = za.y + zb.y, oy = zb.x - za.x;
        const cpx w = rs_tw[32 * i + l];  // W_N^(l + 32 i)
        const float wr = fmaf(w.x, ox, -w.y * oy), wi = fmaf(w.x, oy, w.y * ox);
        const float xr = ex + wr, xi = ey + wi;
        const float yr = ex - wr, yi = ey - wi;
        const float p = fmaf(xr, xr, xi * xi), q = fmaf(yr, yr, yi * yi);
        Pa[33 * i] = p;
        if constexpr (i == 0) Pb[l0 ? -1 : 0] = q;  // lane 0: the Nyquist bin
        else Pb[-33 * i] = q;
      });
      if (l0) P[M / 2 + TPF / 2] = 4.0f * fmaf(rcv[0].x, rcv[0].x, rcv[0].y * rcv[0].y);
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
      float2 *parts = reinterpret_cast<float2 *>(P + 33 * TPF);
      const int2 li = lane_s[l];
      const unsigned fl = (unsigned)li.x;
      int slot = li.y & 1023;
      const float *pl = P + 33 * l;
      const float2 *wl = lw_s + l;
      // The frame's non-finite check: `tot` accumulates p * 0 over the lane's
      // bins (NaN for a NaN or inf bin, and no overflow), then a ballot.
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
      for (int k = l; k <= M; k += TPF) chk = fmaf(P[pad_bin<TPF>(k)], 0.0f, chk);
      const bool bad = (__ballot_sync(FULL, !isfinite(chk)) & gmask) != 0;
      for (int m = l; m < nmel; m += TPF) {
        const float acc = mel_dot_pad<TPF>(mel_s[m], melw, P, bad);
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
  return align16(size_t(31) * S::TPF * 8) + align16(size_t(S::N) * 4) + align16(size_t(S::RS) * 8) +
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
  cpx *tw2 = reinterpret_cast<cpx *>(sp);  // W_M^(j k1), [k1-1][j]
  sp += align16(size_t(31) * TPF * 8);
  float *win_s = reinterpret_cast<float *>(sp);  // analysis window, natural order
  sp += align16(size_t(N) * 4);
  cpx *rs_tw = reinterpret_cast<cpx *>(sp);  // W_N^(c + 32 s) at 33 s + c
  sp += align16(size_t(S::RS) * 8);
  cpx *bufs = reinterpret_cast<cpx *>(sp);
  sp += size_t(F) * S::FSTRIDE * 8;
  // lanes: band words, lane words, lane-minor weights; else packed weights
  // (the packed rows' descriptors are read from global memory)
  int *band_s = reinterpret_cast<int *>(sp);
  int2 *lane_s = reinterpret_cast<int2 *>(sp + align16(4 * (size_t)nmel));
  float2 *lw_s = reinterpret_cast<float2 *>(sp + align16(4 * (size_t)nmel) + 8 * TPF);
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

  for (int i = tid; i < 31 * TPF; i += S::THREADS) {
    const int k1 = i / TPF + 1, jj = i - (k1 - 1) * TPF;
    tw2[i] = root_q(twq, 2 * jj * k1, N);
  }
  for (int i = tid; i < N / 4; i += S::THREADS) {  // halved: see the header comment
    const float4 w = __ldg(reinterpret_cast<const float4 *>(a.window) + i);
    reinterpret_cast<float4 *>(win_s)[i] = make_float4(0.5f * w.x, 0.5f * w.y, 0.5f * w.z, 0.5f * w.w);
  }
  for (int i = tid; i < S::RS; i += S::THREADS) {
    const int s = i / 33, cc = i - 33 * s;
    rs_tw[i] = cc < 32 ? root_q(twq, cc + 32 * s, N) : cpx{0.0f, 0.0f};
  }
  if (lanes) {
    for (int i = tid; i < nmel; i += S::THREADS) band_s[i] = __ldg(a.mel_band + i);
    for (int i = tid; i < TPF; i += S::THREADS) lane_s[i] = __ldg(a.mel_lane + i);
    for (int i = tid; i < 33 * TPF; i += S::THREADS) lw_s[i] = __ldg(a.mel_lw + i);
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
      const float2 *wb = reinterpret_cast<const float2 *>(win_s) + j;
#pragma unroll
      for (int r = 0; r < 32; r++) {
        const float2 w = wb[TPF * r];
        v[r].x *= w.x;
        v[r].y *= w.y;
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
      const cpx g16 = tw2[15 * TPF + j];  // W_M^(16 j)
      static_for<0, 16>([&](auto ki) {
        constexpr int k = decltype(ki)::value;
        const cpx tt = tw_const<k, 32>(o[k]);
        cpx lo = cadd(e[k], tt), hi = csub(e[k], tt);
        if constexpr (k > 0) {
          const cpx tk = tw2[(k - 1) * TPF + j];
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
      static_for<0, 16>([&](auto ii) {
        constexpr int i = decltype(ii)::value;
        const cpx za = z[i];
        cpx zb;
        if constexpr (i == 0) zb = c0 ? (j0 ? z[31] : z[0]) : rcv[15];
        else zb = c0 ? (j0 ? z[31 - i] : z[32 - i]) : rcv[15 - i];
        const float ex = za.x + zb.x, ey = za.y - zb.y;
        const float ox = za.y + zb.y, oy = zb.x - za.x;
        const cpx w = rs_tw[66 * i + 33 * j0 + col];  // W_N^k
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
      const float2 *wl = lw_s + j;
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
      if (j == TPF - 1) {
        const float p = pl[32];
        const float2 w = wl[32 * TPF];
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

static cudaError_t launch_warp2(const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched) {
  using S = W2Shape;
  const size_t tables = a.mel_lane_ok ? align16(4 * (size_t)a.n_mels) + 8 * 34 * (size_t)S::TPF
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
  const size_t tables = a.mel_lane_ok ? align16(4 * (size_t)a.n_mels) + 8 * 34 * (size_t)S::TPF
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
