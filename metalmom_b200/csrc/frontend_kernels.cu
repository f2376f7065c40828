// Frame kernels for the spectral front end on sm_100a.
//
// One CTA tile = F consecutive frames of one clip; each frame is owned by a
// group of TPF = n_fft/32 threads that synchronise on their own named barrier.
// Per frame:
//   gather + window (float2 loads straight from HBM, padding handled in the
//   index math) -> complex FFT of n_fft/2 points (Stockham, radix-16 stages in
//   registers, exchanges through bank-padded shared memory) -> real split ->
//   |X|^2 -> mode epilogue (spectrum rows, mel rows, or log-mel + per-clip max).
// A second kernel applies the clip-global top_db floor and the DCT-II as a
// register-blocked tile product.
//
// Reference semantics followed (MetalMom, Sources/MetalMomCore):
//   frame count / zero padding   Spectral/STFT.swift:241-254
//   window placement             Spectral/STFT.swift:44-57, Filters/Windows.swift:14-48
//   DFT scaling (plain DFT)      Spectral/STFT.swift:298-329
//   dense mel product            Spectral/MelSpectrogram.swift:127-138
//   power_to_db + top_db         Spectral/Scaling.swift:73-118
//   DCT-II ortho                 Features/MFCC.swift:65-106
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "async_copy.cuh"
#include "fft_radix.cuh"
#include "frame_common.cuh"
#include "kernels.h"

namespace mm {

unsigned encode_max_init() { return enc_f(-INFINITY); }
float decode_max(unsigned u) {
  unsigned b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

// ---------------------------------------------------------------------------
// FFT shape for a real frame of N = 2^LOG2N samples (complex length M = N/2):
// radix-16 stages followed by one radix-RLAST stage when log2(M) % 4 != 0.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int stage_radix(int log2m, int q) { return q < log2m / 4 ? 16 : (1 << (log2m % 4)); }
__host__ __device__ constexpr int stage_ns(int log2m, int q) {
  int ns = 1;
  for (int i = 0; i < q; i++) ns *= stage_radix(log2m, i);
  return ns;
}
// Offset of stage q's twiddles {W_{R*Ns}^(k*r) : r in [1,R), k in [0,Ns)}, stored [r-1][k].
__host__ __device__ constexpr int stage_tw_off(int log2m, int q) {
  int off = 0;
  for (int i = 1; i < q; i++) off += (stage_radix(log2m, i) - 1) * stage_ns(log2m, i);
  return off;
}
__host__ __device__ constexpr int n_stages(int log2m) { return log2m / 4 + ((log2m % 4) ? 1 : 0); }
__host__ __device__ constexpr int tw_count(int log2m) { return stage_tw_off(log2m, n_stages(log2m)); }

template <int LOG2N>
struct Shape {
  static constexpr int N = 1 << LOG2N;
  static constexpr int M = N / 2;
  static constexpr int LOG2M = LOG2N - 1;
  static constexpr int TPF = M / 16;  // threads per frame
  static constexpr int N16 = LOG2M / 4;
  static constexpr int RLAST = 1 << (LOG2M % 4);
  static constexpr int PADM = M + M / 16;
  static constexpr int FSTRIDE = PADM + 1;  // complex slots per frame (odd: spreads banks)
  static constexpr bool TW_SMEM = (M <= 2048);
  static constexpr int TWC = tw_count(LOG2M);
  static constexpr int TWN = M / 2;
};

int stage_twiddle_count(int log2n) { return log2n >= 5 ? tw_count(log2n - 1) : 0; }

template <int LOG2N>
struct Frames;  // frames per CTA tile
template <> struct Frames<5> { static constexpr int F = 128; };
template <> struct Frames<6> { static constexpr int F = 64; };
template <> struct Frames<7> { static constexpr int F = 32; };
template <> struct Frames<8> { static constexpr int F = 32; };
template <> struct Frames<9> { static constexpr int F = 16; };
template <> struct Frames<10> { static constexpr int F = 8; };
template <> struct Frames<11> { static constexpr int F = 8; };
template <> struct Frames<12> { static constexpr int F = 4; };
template <> struct Frames<13> { static constexpr int F = 2; };
template <> struct Frames<14> { static constexpr int F = 1; };
template <> struct Frames<15> { static constexpr int F = 1; };

// Launch variants of the frame kernel (picked per n_fft by the autotuner):
//   V0: the default tile, 1024 threads' worth of registers per SM (<= 64 regs);
//   V1: 256-thread CTAs, 3 per SM (<= 85 regs);  V2: 256-thread CTAs, 2 per SM (<= 128 regs).
template <int LOG2N, int V>
struct Cfg {
  static constexpr int TPF = Shape<LOG2N>::TPF;
  static constexpr int F = V == 0 ? Frames<LOG2N>::F : (TPF >= 256 ? 1 : 256 / TPF);
  static constexpr int THREADS = TPF * F;
  static constexpr int BUDGET = V == 0 ? 1024 : (V == 1 ? 768 : 512);
  static constexpr int MINB = BUDGET / THREADS > 0 ? BUDGET / THREADS : 1;
};

__host__ __device__ constexpr bool tunable(int log2n, int mode, int pw) {
  return (mode == MODE_MELDB || (mode == MODE_MEL && pw == 0)) && log2n >= 8 && log2n <= 13;
}

int frame_variants(int log2n, int mode, int power_is_2) {
  if (mode == MODE_MELDB && warp_frames_per_tile(log2n) > 0) return 4;
  return tunable(log2n, mode, power_is_2 ? 0 : 1) ? 3 : 1;
}

template <int LOG2N>
static int frames_for(int v) {
  return v == 1 ? Cfg<LOG2N, 1>::F : (v == 2 ? Cfg<LOG2N, 2>::F : Cfg<LOG2N, 0>::F);
}

int frames_per_tile(int log2n, int variant) {
  if (variant == kDftVariant) return 128;
  if (variant == kTcVariant && log2n == 11) return kTcFramesPerTile;
  if (variant == kWarpVariant && warp_frames_per_tile(log2n) > 0) return warp_frames_per_tile(log2n);
  switch (log2n) {
    case 5: return frames_for<5>(variant);
    case 6: return frames_for<6>(variant);
    case 7: return frames_for<7>(variant);
    case 8: return frames_for<8>(variant);
    case 9: return frames_for<9>(variant);
    case 10: return frames_for<10>(variant);
    case 11: return frames_for<11>(variant);
    case 12: return frames_for<12>(variant);
    case 13: return frames_for<13>(variant);
    case 14: return frames_for<14>(variant);
    case 15: return frames_for<15>(variant);
    default: return 128;  // tiny kernel (n_fft <= 16)
  }
}

// Dynamic shared memory layout of frontend_kernel (host and device agree):
//   [mel_info n_mels x int4][mel weights][red 32 f][bad F i][tws][twn][buf F x FSTRIDE cpx]
template <int LOG2N, int F>
__host__ __device__ constexpr size_t fixed_smem_bytes() {
  using S = Shape<LOG2N>;
  return 128 + align16(F * 4) +
         (S::TW_SMEM ? align16(size_t(S::TWC) * 8) + align16(size_t(S::TWN) * 8) : 0) +
         size_t(F) * S::FSTRIDE * 8;
}

// ---------------------------------------------------------------------------
// main frame kernel, n_fft = 2^LOG2N with LOG2N in [5, 15]
// ---------------------------------------------------------------------------
// MODE_COMPLEX leaves the tile loop right after writing its bins, so the
// power epilogues that follow are unreachable in that instantiation.
#pragma nv_diag_suppress 128
template <int LOG2N, int V, int MODE, int PW>
__global__ void __launch_bounds__(Cfg<LOG2N, V>::THREADS, Cfg<LOG2N, V>::MINB)
frontend_kernel(FrontArgs a) {
  using S = Shape<LOG2N>;
  constexpr int F = Cfg<LOG2N, V>::F;
  constexpr int N = S::N, M = S::M, TPF = S::TPF, THREADS = TPF * F;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nmel = mode_has_mel(MODE) ? a.n_mels : 0;
  const bool mel_in_smem = mode_has_mel(MODE) && a.mel_nnz <= kMelSmemMax;
  unsigned char *sp = smem;
  int4 *mel_s = reinterpret_cast<int4 *>(sp);
  sp += 16 * (size_t)nmel;
  float *melw_s = reinterpret_cast<float *>(sp);
  if (mel_in_smem) sp += align16(4 * (size_t)a.mel_nnz);
  sp += 128;  // (a reserved 128-byte slot of the layout)
  int *bad_s = reinterpret_cast<int *>(sp);
  sp += align16(F * 4);
  cpx *tws_s = reinterpret_cast<cpx *>(sp);
  if constexpr (S::TW_SMEM) sp += align16(size_t(S::TWC) * 8);
  cpx *twn_s = reinterpret_cast<cpx *>(sp);
  if constexpr (S::TW_SMEM) sp += align16(size_t(S::TWN) * 8);
  cpx *buf = reinterpret_cast<cpx *>(sp);

  const int tid = threadIdx.x;
  const int f = tid / TPF;
  const int j = tid - f * TPF;

  if constexpr (S::TW_SMEM) {
    for (int i = tid; i < S::TWC; i += THREADS) tws_s[i] = ldc(a.tw_stage + i);
    for (int i = tid; i < S::TWN; i += THREADS) twn_s[i] = ldc(a.tw_split + i);
  }
  for (int i = tid; i < nmel; i += THREADS) mel_s[i] = __ldg(a.mel_info + i);
  if (mel_in_smem)
    for (int i = tid; i < a.mel_nnz; i += THREADS) melw_s[i] = __ldg(a.mel_pw + i);
  const cpx *tws = S::TW_SMEM ? tws_s : reinterpret_cast<const cpx *>(a.tw_stage);
  const cpx *twn = S::TW_SMEM ? twn_s : reinterpret_cast<const cpx *>(a.tw_split);
  const float *melw = mel_in_smem ? melw_s : a.mel_pw;
  __syncthreads();

  cpx *fb = buf + f * S::FSTRIDE;
  float *P = reinterpret_cast<float *>(fb);

  for (int tile = blockIdx.x; tile < a.total_tiles; tile += gridDim.x) {
    const int c = __ldg(a.tile_clip + tile);
    const ClipDesc cd = load_clip(a.clips + c);
    const int t0 = (tile - cd.tile_base) * F;
    const int t = t0 + f;
    // Log-mel frame groups that fill whole warps work independently: an
    // out-of-range frame skips the tile (its group's barriers are its own).
    if (MODE == MODE_MELDB && TPF >= 32 && t >= cd.n_frames) continue;
    const long long s0 = (long long)t * a.hop - a.pad;
    const float *sig = a.signal + cd.sig_off;

    // ---- gather: z[n] = (x[2n] w[2n], x[2n+1] w[2n+1]) for n = j + r*M/16
    cpx v[16];
    if (s0 >= 0 && s0 + N <= cd.length) {
      const float *base = sig + s0 + 2 * j;
      const float *wb = a.window + 2 * j;
      if (((cd.sig_off + s0) & 1) == 0) {
#pragma unroll
        for (int r = 0; r < 16; r++) {
          const float2 x = __ldg(reinterpret_cast<const float2 *>(base + r * (N / 16)));
          const float2 w = __ldg(reinterpret_cast<const float2 *>(wb + r * (N / 16)));
          v[r] = {x.x * w.x, x.y * w.y};
        }
      } else {
#pragma unroll
        for (int r = 0; r < 16; r++) {
          const float2 w = __ldg(reinterpret_cast<const float2 *>(wb + r * (N / 16)));
          v[r] = {__ldg(base + r * (N / 16)) * w.x, __ldg(base + r * (N / 16) + 1) * w.y};
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < 16; r++) {
        const int n0 = 2 * j + r * (N / 16);
        const float2 w = __ldg(reinterpret_cast<const float2 *>(a.window + n0));
        v[r] = {sample_at(sig, s0 + n0, cd.length, a.pad_mode) * w.x,
                sample_at(sig, s0 + n0 + 1, cd.length, a.pad_mode) * w.y};
      }
    }

    // ---- stage 0: radix 16, Ns = 1 (no twiddles)
    dft16(v);
    frame_sync<TPF>(f);  // the previous tile's epilogue has finished with fb
#pragma unroll
    for (int r = 0; r < 16; r++) fb[padx(j * 16 + r)] = v[r];
    frame_sync<TPF>(f);

    // ---- radix-16 stages 1 .. N16-1
#pragma unroll
    for (int q = 1; q < S::N16; q++) {
      const int Ns = 1 << (4 * q);
      const int k = j & (Ns - 1);
      const cpx *tw = tws + stage_tw_off(S::LOG2M, q) + k;
#pragma unroll
      for (int r = 0; r < 16; r++) v[r] = fb[padx(j + r * (M / 16))];
#pragma unroll
      for (int r = 1; r < 16; r++) v[r] = cmul(v[r], tw[(r - 1) * Ns]);
      dft16(v);
      frame_sync<TPF>(f);
      const int base = (j - k) * 16 + k;
#pragma unroll
      for (int r = 0; r < 16; r++) fb[padx(base + r * Ns)] = v[r];
      frame_sync<TPF>(f);
    }

    // ---- trailing radix-R stage (in place: each thread rewrites what it read)
    if constexpr (S::RLAST > 1) {
      constexpr int R = S::RLAST, B = 16 / R, Ns = M / R;
      const cpx *tw = tws + stage_tw_off(S::LOG2M, S::N16);
#pragma unroll
      for (int i = 0; i < B; i++) {
        const int b = j + i * TPF;
#pragma unroll
        for (int qq = 0; qq < R; qq++) v[i * R + qq] = fb[padx(b + qq * Ns)];
#pragma unroll
        for (int qq = 1; qq < R; qq++) v[i * R + qq] = cmul(v[i * R + qq], tw[(qq - 1) * Ns + b]);
        dft<R>(v + i * R);
#pragma unroll
        for (int qq = 0; qq < R; qq++) fb[padx(b + qq * Ns)] = v[i * R + qq];
      }
      frame_sync<TPF>(f);
    }

    // ---- real split: X[k] = E + W^k O, X[M-k] = conj(E - W^k O)
    if constexpr (MODE == MODE_COMPLEX) {
      // the bins themselves, staged in the frame buffer (bin k at slot k) and
      // written [k][t] by the whole CTA; DC and Nyquist carry no imaginary part
      cpx xa[8], xb[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int k = j + i * TPF;
        if (k == 0) {
          const cpx z = fb[0];
          xa[i] = {z.x + z.y, 0.0f};
          xb[i] = {z.x - z.y, 0.0f};
        } else {
          const cpx za = fb[padx(k)], zb = fb[padx(M - k)];
          const cpx E = {0.5f * (za.x + zb.x), 0.5f * (za.y - zb.y)};
          const cpx O = {0.5f * (za.y + zb.y), -0.5f * (za.x - zb.x)};
          const cpx WO = cmul(twn[k], O);
          xa[i] = {E.x + WO.x, E.y + WO.y};
          xb[i] = {E.x - WO.x, -(E.y - WO.y)};
        }
      }
      cpx xmid = {0.0f, 0.0f};
      if (j == 0) {
        const cpx z = fb[padx(M / 2)];
        xmid = {z.x, -z.y};
      }
      frame_sync<TPF>(f);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int k = j + i * TPF;
        fb[k] = xa[i];
        fb[M - k] = xb[i];
      }
      if (j == 0) fb[M / 2] = xmid;
      __syncthreads();
      const long long T = cd.n_frames;
      const cpx *X0 = buf;
      float2 *dst = reinterpret_cast<float2 *>(a.out + cd.out_off);
      for (int it = tid; it < F * (M + 1); it += THREADS) {
        const int fi = it % F, k = it / F;
        const int tt = t0 + fi;
        if (tt < cd.n_frames) {
          const cpx x = X0[fi * S::FSTRIDE + k];
          dst[(long long)k * T + tt] = make_float2(x.x, x.y);
        }
      }
      __syncthreads();  // the next tile overwrites buf
      continue;
    }
    float pa[8], pb[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int k = j + i * TPF;
      if (k == 0) {
        const cpx z = fb[0];
        const float dc = z.x + z.y, ny = z.x - z.y;
        pa[i] = dc * dc;
        pb[i] = ny * ny;
      } else {
        const cpx za = fb[padx(k)], zb = fb[padx(M - k)];
        const cpx E = {0.5f * (za.x + zb.x), 0.5f * (za.y - zb.y)};
        const cpx O = {0.5f * (za.y + zb.y), -0.5f * (za.x - zb.x)};
        const cpx WO = cmul(twn[k], O);
        const float xr = E.x + WO.x, xi = E.y + WO.y;
        const float yr = E.x - WO.x, yi = E.y - WO.y;
        pa[i] = xr * xr + xi * xi;
        pb[i] = yr * yr + yi * yi;
      }
    }
    float pmid = 0.0f;
    if (j == 0) {
      const cpx z = fb[padx(M / 2)];
      pmid = z.x * z.x + z.y * z.y;
    }
    frame_sync<TPF>(f);
    // the log-mel epilogue's filterbank walk reads the spectrum padded (bin k
    // at k + min(k / 32, TW - 1), TW = TPF / 2 walking threads of 32 bins), so
    // that its 32 bins per thread are conflict-free rows of 33
    constexpr int TW = TPF / 2;
    const bool walk = MODE == MODE_MELDB && a.mel_lane_ok;
    auto pk = [&](int k) { return walk ? k + min(k >> 5, TW - 1) : k; };
    float chk = 0.0f;  // sum of this thread's |X|^power * 0: NaN iff one term is not finite
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int k = j + i * TPF;
      const float x = apply_power<PW>(pa[i], a.power);
      const float y = apply_power<PW>(pb[i], a.power);
      P[pk(k)] = x;
      P[pk(M - k)] = y;
      chk = fmaf(x, 0.0f, fmaf(y, 0.0f, chk));
    }
    if (j == 0) {
      const float x = apply_power<PW>(pmid, a.power);
      P[pk(M / 2)] = x;
      chk = fmaf(x, 0.0f, chk);
    }
    const bool bad = frame_sync_or<TPF>(f, !isfinite(chk));

    if constexpr (MODE == MODE_MELDB) {
      // frame-local epilogue: log-mel row of this frame + running clip max
      const bool valid = t < cd.n_frames;
      float vmax = -INFINITY;
      float *dst = a.out + (cd.frame_off + t) * (long long)a.n_mels;
      const float ref_db = 10.0f * log10f(a.ref);
      if (walk) {
        // the warp kernel's filterbank walk (tables at build_mel_lane_kernel):
        // thread j < TW sums its 32 bins into part slots, segment heads take
        // the parts of the threads they run into, a band is two slot reads
        float2 *parts = reinterpret_cast<float2 *>(P + 33 * TW);
        int hslot = 0, chain = 0;
        if (j < TW) {
          const int2 li = __ldg(a.mel_lane + j);
          const unsigned fl = (unsigned)li.x;
          int slot = li.y & 1023;
          const float *pl = P + 33 * j;
          float R = 0.0f, Fs = 0.0f;
#pragma unroll
          for (int b = 0; b < 32; b++) {
            const float p = pl[b];
            const float2 w = __ldg(a.mel_lw + b * TW + j);
            R = fmaf(w.x, p, R);
            Fs = fmaf(w.y, p, Fs);
            if (fl & (1u << b)) {
              parts[slot++] = make_float2(R, Fs);
              R = 0.0f;
              Fs = 0.0f;
            }
          }
          if (j == TW - 1) {
            const float p = pl[32];
            const float2 w = __ldg(a.mel_lw + 32 * TW + j);
            parts[slot] = make_float2(fmaf(w.x, p, R), fmaf(w.y, p, Fs));
          }
          if (j == 0) parts[li.y >> 16] = make_float2(0.0f, 0.0f);  // the empty segments' slot
          hslot = j == TW - 1 ? slot : slot - 1;
          chain = (li.y >> 10) & 63;
        }
        frame_sync<TPF>(f);
        if (chain) {
          float2 hv = parts[hslot];
          for (int q = 1; q <= chain; q++) {
            const float2 pv = parts[hslot + q];
            hv.x += pv.x;
            hv.y += pv.y;
          }
          parts[hslot] = hv;
        }
        frame_sync<TPF>(f);
        for (int m = j; m < a.n_mels; m += TPF) {
          const int bw = __ldg(a.mel_band + m);
          float acc = parts[bw & 4095].x + parts[(bw >> 12) & 4095].y;
          if (((bw >> 24) & 1) || bad) acc = __int_as_float(0x7fc00000);
          const float v = db10_frame(acc, a.amin, ref_db);
          if (valid) dst[m] = v;
          vmax = fmaxf(vmax, v);
        }
      } else {
        for (int m = j; m < a.n_mels; m += TPF) {
          const float acc = mel_dot(mel_s[m], melw, P, bad);
          const float v = db10_frame(acc, a.amin, ref_db);
          if (valid) dst[m] = v;
          vmax = fmaxf(vmax, v);
        }
      }
      if (!valid) vmax = -INFINITY;
      constexpr int W = TPF < 32 ? TPF : 32;
#pragma unroll
      for (int o = W / 2; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      if ((j & (W - 1)) == 0 && vmax > -INFINITY) atomicMax(a.clip_max + c, enc_f(vmax));
    } else {
      // CTA-wide epilogues write [rows][T] blocks: F consecutive frames per row
      if (j == 0) bad_s[f] = bad ? 1 : 0;
      __syncthreads();
      const long long T = cd.n_frames;
      const float *P0 = reinterpret_cast<const float *>(buf);
      constexpr int FS = 2 * S::FSTRIDE;
      if constexpr (MODE == MODE_SPECTRUM) {
        for (int it = tid; it < F * (M + 1); it += THREADS) {
          const int fi = it % F, k = it / F;
          const int tt = t0 + fi;
          if (tt < cd.n_frames) a.out[cd.out_off + (long long)k * T + tt] = P0[fi * FS + k];
        }
      } else {
        for (int it = tid; it < F * a.n_mels; it += THREADS) {
          const int fi = it % F, m = it / F;
          const int tt = t0 + fi;
          if (tt >= cd.n_frames) continue;
          a.out[cd.out_off + (long long)m * T + tt] = mel_dot(mel_s[m], melw, P0 + fi * FS, bad_s[fi] != 0);
        }
      }
      __syncthreads();  // the next tile overwrites buf
    }
  }
}
#pragma nv_diag_default 128

// ---------------------------------------------------------------------------
// tiny frames (n_fft <= 16): direct DFT, one thread per frame
// ---------------------------------------------------------------------------
template <int MODE, int PW>
__global__ void __launch_bounds__(128) frontend_tiny_kernel(FrontArgs a, int n_fft) {
  constexpr int F = 128, THREADS = 128, PST = 9;
  constexpr int CW = (MODE == MODE_COMPLEX) ? 2 : 1;  // floats per bin
  __shared__ __align__(8) float P_s[F * PST * CW];
  __shared__ int bad_s[F];
  __shared__ float red_s[32];
  extern __shared__ __align__(16) unsigned char smem[];
  const int nmel = mode_has_mel(MODE) ? a.n_mels : 0;
  int4 *mel_s = reinterpret_cast<int4 *>(smem);
  float *melw_s = reinterpret_cast<float *>(smem + 16 * (size_t)nmel);
  const bool mel_in_smem = mode_has_mel(MODE) && a.mel_nnz <= kMelSmemMax;
  const int tid = threadIdx.x;
  for (int i = tid; i < nmel; i += THREADS) mel_s[i] = __ldg(a.mel_info + i);
  if (mel_in_smem)
    for (int i = tid; i < a.mel_nnz; i += THREADS) melw_s[i] = __ldg(a.mel_pw + i);
  const float *melw = mel_in_smem ? melw_s : a.mel_pw;
  const int nfreq = n_fft / 2 + 1;
  for (int tile = blockIdx.x; tile < a.total_tiles; tile += gridDim.x) {
    const int c = __ldg(a.tile_clip + tile);
    const ClipDesc cd = load_clip(a.clips + c);
    const int t0 = (tile - cd.tile_base) * F;
    const long long s0 = (long long)(t0 + tid) * a.hop - a.pad;
    const float *sig = a.signal + cd.sig_off;
    float xw[16];
#pragma unroll
    for (int n = 0; n < 16; n++)
      xw[n] = (n < n_fft) ? sample_at(sig, s0 + n, cd.length, a.pad_mode) * __ldg(a.window + n) : 0.0f;
    if constexpr (MODE == MODE_COMPLEX) {
      float2 x[PST];
#pragma unroll
      for (int k = 0; k < PST; k++) {
        float re = 0.0f, im = 0.0f;
        if (k < nfreq) {
          for (int n = 0; n < n_fft; n++) {
            const float2 w = __ldg(a.tw_tiny + ((n * k) % n_fft));
            re = fmaf(xw[n], w.x, re);
            im = fmaf(xw[n], w.y, im);
          }
        }
        if (k == 0 || 2 * k == n_fft) im = 0.0f;  // DC and Nyquist are real
        x[k] = make_float2(re, im);
      }
      __syncthreads();
      float2 *X_s = reinterpret_cast<float2 *>(P_s);
#pragma unroll
      for (int k = 0; k < PST; k++) X_s[tid * PST + k] = x[k];
      __syncthreads();
      const long long T = cd.n_frames;
      float2 *dst = reinterpret_cast<float2 *>(a.out + cd.out_off);
      for (int it = tid; it < F * nfreq; it += THREADS) {
        const int fi = it % F, k = it / F;
        const int tt = t0 + fi;
        if (tt < cd.n_frames) dst[(long long)k * T + tt] = X_s[fi * PST + k];
      }
      continue;
    }
    float p[PST];
    float chk = 0.0f;
#pragma unroll
    for (int k = 0; k < PST; k++) {
      float re = 0.0f, im = 0.0f;
      if (k < nfreq) {
        for (int n = 0; n < n_fft; n++) {
          const float2 w = __ldg(a.tw_tiny + ((n * k) % n_fft));
          re = fmaf(xw[n], w.x, re);
          im = fmaf(xw[n], w.y, im);
        }
      }
      p[k] = apply_power<PW>(re * re + im * im, a.power);
      if (k < nfreq) chk = fmaf(p[k], 0.0f, chk);  // NaN iff a bin is not finite
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PST; k++) P_s[tid * PST + k] = p[k];
    bad_s[tid] = !isfinite(chk);
    __syncthreads();
    const long long T = cd.n_frames;
    if constexpr (MODE == MODE_SPECTRUM) {
      for (int it = tid; it < F * nfreq; it += THREADS) {
        const int fi = it % F, k = it / F;
        const int tt = t0 + fi;
        if (tt < cd.n_frames) a.out[cd.out_off + (long long)k * T + tt] = P_s[fi * PST + k];
      }
    } else if constexpr (MODE == MODE_MEL) {
      for (int it = tid; it < F * a.n_mels; it += THREADS) {
        const int fi = it % F, m = it / F;
        const int tt = t0 + fi;
        if (tt < cd.n_frames)
          a.out[cd.out_off + (long long)m * T + tt] = mel_dot(mel_s[m], melw, P_s + fi * PST, bad_s[fi] != 0);
      }
    } else {
      float vmax = -INFINITY;
      for (int it = tid; it < F * a.n_mels; it += THREADS) {
        const int fi = it / a.n_mels, m = it - fi * a.n_mels;
        const int tt = t0 + fi;
        if (tt >= cd.n_frames) continue;
        const float acc = mel_dot(mel_s[m], melw, P_s + fi * PST, bad_s[fi] != 0);
        const float v = db10_frame(acc, a.amin, 10.0f * log10f(a.ref));
        a.out[(cd.frame_off + tt) * (long long)a.n_mels + m] = v;
        vmax = fmaxf(vmax, v);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      if ((tid & 31) == 0) red_s[tid >> 5] = vmax;
      __syncthreads();
      if (tid < 32) {
        float v = (tid < THREADS / 32) ? red_s[tid] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (tid == 0 && v > -INFINITY) atomicMax(a.clip_max + c, enc_f(v));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// top_db floor + DCT-II over the frame-major log-mel: per tile of 64 frames of
// one clip, out[k][t] = sum_n B[k][n] * max(D[t][n], max_db - top_db).
// 256 threads = 64 frames x 4 coefficient groups of KQ coefficients each.
// ---------------------------------------------------------------------------
constexpr int kDctMC = 64;        // mel chunk
constexpr int kDctTS = kDctMC + 4;  // tile row stride (floats): float4 rows, conflict-free
constexpr int kDctKC = 32;        // coefficient chunk

template <int KQ>
__global__ void __launch_bounds__(256) dct_kernel(DctArgs a) {
  constexpr int TT = kDctTile;
  __shared__ __align__(16) float tile[TT * kDctTS];
  __shared__ __align__(16) float bas[4 * KQ * kDctMC];
  const int tid = threadIdx.x;
  const int fr = tid & (TT - 1), kg = tid / TT;
  for (int ti = blockIdx.x; ti < a.total_tiles; ti += gridDim.x) {
    const int c = __ldg(a.tile_clip + ti);
    const ClipDesc cd = load_clip(a.clips + c);
    const int tf = __ldg(a.tile_first + ti);
    const int nt = min(TT, cd.n_frames - tf);
    const bool floor_on = a.top_db > 0.0f;
    const float thr = floor_on ? dec_f(__ldg(a.clip_max + c)) - a.top_db : 0.0f;
    const float *src = a.mel_db + (cd.frame_off + tf) * (long long)a.n_mels;
    const bool vec4 = (a.n_mels & 3) == 0;  // mel_db is 256-byte aligned, rows n_mels floats
    const long long T = cd.n_frames;
    for (int kc = 0; kc < a.n_mfcc; kc += 4 * KQ) {
      float acc[KQ];
#pragma unroll
      for (int q = 0; q < KQ; q++) acc[q] = 0.0f;
      for (int mc = 0; mc < a.n_mels; mc += kDctMC) {
        const int mw = min(kDctMC, a.n_mels - mc);
        __syncthreads();
        if (vec4) {
          // rows of the frame-major log-mel are 16-byte aligned: 4 float4 per thread, loads first
          float4 x[TT * kDctMC / 4 / 256];
#pragma unroll
          for (int u = 0; u < TT * kDctMC / 4 / 256; u++) {
            const int i = tid + 256 * u;
            const int r = i / (kDctMC / 4), c4 = i - r * (kDctMC / 4);
            x[u] = (r < nt && 4 * c4 < mw)
                       ? __ldg(reinterpret_cast<const float4 *>(src + (long long)r * a.n_mels + mc) + c4)
                       : make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
          for (int u = 0; u < TT * kDctMC / 4 / 256; u++) {
            const int i = tid + 256 * u;
            const int r = i / (kDctMC / 4), c4 = i - r * (kDctMC / 4);
            float4 v = x[u];
            if (floor_on && r < nt && 4 * c4 < mw) {
              v.x = vthr(v.x, thr);
              v.y = vthr(v.y, thr);
              v.z = vthr(v.z, thr);
              v.w = vthr(v.w, thr);
            }
            *reinterpret_cast<float4 *>(tile + r * kDctTS + 4 * c4) = v;
          }
        } else {
          float x[TT * kDctMC / 256];
#pragma unroll
          for (int u = 0; u < TT * kDctMC / 256; u++) {
            const int i = tid + 256 * u;
            const int r = i / kDctMC, col = i - r * kDctMC;
            x[u] = (r < nt && col < mw) ? __ldg(src + (long long)r * a.n_mels + mc + col) : 0.0f;
          }
#pragma unroll
          for (int u = 0; u < TT * kDctMC / 256; u++) {
            const int i = tid + 256 * u;
            const int r = i / kDctMC, col = i - r * kDctMC;
            float v = x[u];
            if (floor_on && r < nt && col < mw) v = vthr(v, thr);
            tile[r * kDctTS + col] = v;
          }
        }
        for (int i = tid; i < 4 * KQ * kDctMC; i += 256) {
          const int k = i / kDctMC, col = i - k * kDctMC;
          const int kk = kc + k;
          bas[i] = (kk < a.n_mfcc && col < mw) ? __ldg(a.basis + (long long)kk * a.n_mels + mc + col) : 0.0f;
        }
        __syncthreads();
        const float4 *trow = reinterpret_cast<const float4 *>(tile + fr * kDctTS);
        const float4 *brow = reinterpret_cast<const float4 *>(bas + kg * KQ * kDctMC);
#pragma unroll 4
        for (int n4 = 0; n4 < kDctMC / 4; n4++) {
          const float4 d = trow[n4];
#pragma unroll
          for (int q = 0; q < KQ; q++) {
            const float4 b = brow[q * (kDctMC / 4) + n4];
            acc[q] = fmaf(b.x, d.x, acc[q]);
            acc[q] = fmaf(b.y, d.y, acc[q]);
            acc[q] = fmaf(b.z, d.z, acc[q]);
            acc[q] = fmaf(b.w, d.w, acc[q]);
          }
        }
      }
      if (fr < nt) {
#pragma unroll
        for (int q = 0; q < KQ; q++) {
          const int k = kc + kg * KQ + q;
          if (k < a.n_mfcc) a.out[cd.out_off + (long long)k * T + tf + fr] = acc[q];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// dB scaling over a flat array (mm_power_to_db / mm_amplitude_to_db)
// ---------------------------------------------------------------------------
// ref_slot (optional): {encoded max of x, NaN flag} written by db_ref_kernel;
// the reference value is then max(x) (NaN when x holds one), as ref=np.max.
__global__ void __launch_bounds__(256) db_pass1_kernel(const float *x, float *y, long long n,
                                                       float mult, float amin, float ref,
                                                       const unsigned *ref_slot, unsigned *slot) {
  __shared__ float red[8];
  if (ref_slot) ref = ref_slot[1] ? __int_as_float(0x7fc00000) : dec_f(ref_slot[0]);
  float vmax = -INFINITY;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float v = mult * log10f(vthr(x[i], amin) / ref);
    y[i] = v;
    vmax = fmaxf(vmax, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < 8 ? red[threadIdx.x] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0 && v > -INFINITY) atomicMax(slot, enc_f(v));
  }
}

__global__ void __launch_bounds__(256) db_ref_kernel(const float *x, long long n, unsigned *ref_slot) {
  __shared__ float red[8];
  float vmax = -INFINITY;
  bool nan = false;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const float v = x[i];
    nan |= isnan(v);
    vmax = fmaxf(vmax, v);
  }
  if (__syncthreads_or(nan) && threadIdx.x == 0) atomicOr(ref_slot + 1, 1u);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < 8 ? red[threadIdx.x] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) atomicMax(ref_slot, enc_f(v));
  }
}

__global__ void __launch_bounds__(256) db_pass2_kernel(float *y, long long n, float top_db,
                                                       const unsigned *slot) {
  const float thr = dec_f(*slot) - top_db;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
    y[i] = vthr(y[i], thr);
}

__global__ void fill_pattern_kernel(float *p, long long n) {
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    unsigned h = (unsigned)i * 2654435761u;
    h ^= h >> 16;
    h *= 2246822519u;
    h ^= h >> 13;
    p[i] = (float)(h & 0xffffff) / 16777216.0f - 0.5f;
  }
}

__global__ void fill_u32_kernel(unsigned *p, unsigned v, long long n) {
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256) p[i] = v;
}

// ---------------------------------------------------------------------------
// table builders: float64 arithmetic on the device, rounded once to float32
// ---------------------------------------------------------------------------
__global__ void build_window_kernel(float *w, int n_fft, int win, int zero) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n_fft) return;
  double v = 0.0;
  if (!zero && win > 0) {
    long long idx;
    if (win < n_fft) idx = (long long)n - (n_fft - win) / 2;
    else if (win > n_fft) idx = (long long)n + (win - n_fft) / 2;
    else idx = n;
    if (idx >= 0 && idx < win) v = (win == 1) ? 1.0 : 0.5 - 0.5 * cospi(2.0 * (double)idx / (double)win);
  }
  w[n] = (float)v;
}

// exp(-2 pi i t / period) for t = k*r, r in [1,R), k in [0,Ns): stored [r-1][k]
__global__ void build_stage_tw_kernel(float2 *tw, int R, int Ns) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (R - 1) * Ns) return;
  const int r = i / Ns + 1, k = i - (r - 1) * Ns;
  const long long period = (long long)R * Ns;
  const long long t = ((long long)k * r) % period;
  double s, c;
  sincospi(-2.0 * (double)t / (double)period, &s, &c);
  tw[i] = make_float2((float)c, (float)s);
}

__global__ void build_roots_kernel(float2 *tw, int count, int period) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  double s, c;
  sincospi(-2.0 * (double)t / (double)period, &s, &c);
  tw[t] = make_float2((float)c, (float)s);
}

__device__ double hz_to_mel_d(double hz) {
  const double f_sp = 200.0 / 3.0, min_log_mel = 1000.0 / f_sp, logstep = log(6.4) / 27.0;
  double mel = hz / f_sp;
  if (hz >= 1000.0) mel = min_log_mel + log(hz / 1000.0) / logstep;
  return mel;
}
__device__ double mel_to_hz_d(double mel) {
  const double f_sp = 200.0 / 3.0, min_log_mel = 1000.0 / f_sp, logstep = log(6.4) / 27.0;
  if (mel < min_log_mel) return mel * f_sp;
  return 1000.0 * exp((mel - min_log_mel) * logstep);
}

// Dense Slaney filterbank, one thread per (mel, bin) (FilterBank.swift:23-73).
__global__ void build_mel_kernel(float *W, int sr, int n_fft, int n_mels, double fmin, double fmax) {
  const int nfreq = n_fft / 2 + 1;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)n_mels * nfreq) return;
  const int m = (int)(i / nfreq), k = (int)(i - (long long)m * nfreq);
  const double lo = hz_to_mel_d(fmin), hi = hz_to_mel_d(fmax);
  const double step = (hi - lo) / (double)(n_mels + 1);
  const double fl = mel_to_hz_d(lo + m * step);
  const double fc = mel_to_hz_d(lo + (m + 1) * step);
  const double fr = mel_to_hz_d(lo + (m + 2) * step);
  const double f = (double)k * (double)sr / (double)n_fft;
  double w = 0.0;
  if (f >= fl && f <= fc && fc != fl) w = (f - fl) / (fc - fl);
  else if (f > fc && f <= fr && fr != fc) w = (fr - f) / (fr - fc);
  const double enorm = 2.0 / (fr - fl);
  W[i] = (float)(w * enorm);
}

// Per-mel nonzero range of the dense filterbank + NaN-row flag (z = count for now).
__global__ void build_mel_info_kernel(int4 *info, const float *W, int n_mels, int nfreq) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_mels) return;
  const float *row = W + (long long)m * nfreq;
  int first = -1, last = -1, nan_row = 0;
  for (int k = 0; k < nfreq; k++) {
    const float w = row[k];
    if (isnan(w)) nan_row = 1;
    if (w != 0.0f) {
      if (first < 0) first = k;
      last = k;
    }
  }
  if (first < 0) info[m] = make_int4(0, 0, 0, nan_row);
  else info[m] = make_int4(first, last - first + 1, 0, nan_row);
}

// Exclusive prefix sum of the row lengths into info[m].z; total into *nnz.
__global__ void mel_offsets_kernel(int4 *info, int n_mels, int *nnz) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int off = 0;
  for (int m = 0; m < n_mels; m++) {
    info[m].z = off;
    off += info[m].y;
  }
  *nnz = off;
}

// Per-bin split of the dense filterbank.  A Slaney bin feeds at most two
// consecutive bands (the falling edge of band s-1 and the rising edge of band
// s): w2[k] = (weight of band s, weight of band s-1), bin_seg[k] = s; a bin
// with one band m gets (weight, 0) and s = m; -1: no band; -2: a pattern the
// split cannot express.
__global__ void build_mel_bins_kernel(float2 *w2, int *bin_seg, const float *W, int n_mels, int nfreq) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nfreq) return;
  int first = -1, last = -1, cnt = 0;
  for (int m = 0; m < n_mels; m++) {
    if (W[(long long)m * nfreq + k] != 0.0f) {  // NaN counts as nonzero
      if (first < 0) first = m;
      last = m;
      cnt++;
    }
  }
  if (cnt == 0) {
    w2[k] = make_float2(0.0f, 0.0f);
    bin_seg[k] = -1;
  } else if (cnt == 1) {
    w2[k] = make_float2(W[(long long)first * nfreq + k], 0.0f);
    bin_seg[k] = first;
  } else if (cnt == 2 && last == first + 1) {
    w2[k] = make_float2(W[(long long)last * nfreq + k], W[(long long)first * nfreq + k]);
    bin_seg[k] = last;
  } else {
    w2[k] = make_float2(0.0f, 0.0f);
    bin_seg[k] = -2;
  }
}

// Segment table from bin_seg (one thread): seg[s].x = first bin of segment s
// (empty segments start where the next one does), seg[n_mels].x = one past the
// last bin that feeds a band, seg[s].y = NaN flag of band s.  ok[1] = 1 when
// every bin is expressible and the band of the bins never decreases.
__global__ void build_mel_seg_kernel(int2 *seg, const int *bin_seg, const int4 *info, int n_mels, int nfreq,
                                     int *ok) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int prev = -1, good = 1, end = 0;
  for (int s = 0; s <= n_mels; s++) seg[s] = make_int2(-1, s < n_mels ? info[s].w : 0);
  for (int k = 0; k < nfreq; k++) {
    const int s = bin_seg[k];
    if (s == -2) good = 0;
    if (s < 0) continue;
    if (s < prev) good = 0;
    if (seg[s].x < 0) seg[s].x = k;
    end = k + 1;
    prev = s;
  }
  seg[n_mels].x = end;
  for (int s = n_mels - 1; s >= 0; s--)
    if (seg[s].x < 0) seg[s].x = seg[s + 1].x;
  ok[1] = good;
}

// Lane tables of the warp kernel's filterbank walk (one thread).  Lane l of a
// frame group owns bins [32 l, 32 l + 32) (the last lane also the Nyquist bin
// M = 32 tpf); it accumulates (R, F) = sum of (w2.x P, w2.y P) and stores the
// pair in the next "part" slot wherever the segment of bin k differs from that
// of bin k+1, and after its last bin.  Parts are numbered lane after lane, so
// the pieces of a segment occupy consecutive slots: its head (the first) and
// the first parts of the following lanes it runs into.  After the walk the
// lane holding a head adds those k continuation parts into it, so each
// segment's sums sit in its head slot and band m = head(m).x + head(m+1).y.
//   lw[b * tpf + l]  = w2[32 l + b], b <= 32 (b = 32: Nyquist, last lane only)
//   lane[l]          = {flush mask over b < 32,
//                       first slot of lane l | k << 10 | zero slot << 16}
//   band[m]          = head slot of segment m | head slot of m+1 << 12 |
//                      NaN flag of band m << 24   (an empty segment: the zero
//                      slot, which the kernel clears every frame)
// ok[2] = 1 when the split holds, every weight is finite and the parts and the
// zero slot fit in `max_slots`.
__global__ void build_mel_lane_kernel(float2 *lw, int2 *lane, int *band, const float2 *w2, const int *bin_seg,
                                      const int2 *seg, int n_mels, int tpf, int max_slots, int *ok) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  ok[2] = 0;
  if (!ok[1] || tpf > 64) return;
  // first(s) | count(s) << 12 during the walk; a segment has one part per
  // lane it touches, so count <= 64 (7 bits) and its chain k = count - 1 <= 63
  for (int m = 0; m < n_mels; m++) band[m] = 0;
  int slot = 0, sid = -1;
  int last_slot[64], last_sid[64];
  // segment of bin k: the band of the last bin at or below k that feeds one
  // (bins with no band carry on the run before them, with zero weights)
  auto next_sid = [&](int k, int cur) { return bin_seg[k] >= 0 ? bin_seg[k] : cur; };
  for (int l = 0; l < tpf; l++) {
    lane[l] = make_int2(0, slot);
    const int last = (l == tpf - 1) ? 32 : 31;
    unsigned mask = 0u;
    for (int b = 0; b <= last; b++) {
      const int k = 32 * l + b;
      sid = next_sid(k, sid);
      if (!isfinite(w2[k].x) || !isfinite(w2[k].y)) return;  // the walk's check needs finite weights
      lw[b * tpf + l] = w2[k];
      const bool flush = (b == last) || next_sid(k + 1, sid) != sid;
      if (!flush) continue;
      if (b < 32) mask |= 1u << b;
      if (sid >= 0) {
        if (slot >= 1023 || sid >= n_mels) return;
        int w = band[sid];
        if (((w >> 12) & 127) == 0) w = slot;  // first part of segment sid
        w += 1 << 12;
        band[sid] = w;
      }
      last_slot[l] = slot;
      last_sid[l] = sid;
      slot++;
    }
    if (l < tpf - 1) lw[32 * tpf + l] = make_float2(0.0f, 0.0f);
    lane[l].x = (int)mask;
  }
  const int zero = slot;
  if (zero + 1 > max_slots) return;
  for (int l = 0; l < tpf; l++) {
    const int s = last_sid[l];
    int k = 0;
    if (s >= 0 && last_slot[l] == (band[s] & 4095)) k = ((band[s] >> 12) & 127) - 1;  // lane l holds the head
    lane[l].y |= (k << 10) | (zero << 16);
  }
  for (int m = 0; m < n_mels; m++) {  // band[m + 1] is still in the walk's form when band[m] is rewritten
    const int hr = ((band[m] >> 12) & 127) ? (band[m] & 4095) : zero;
    const int hf = (m + 1 < n_mels && ((band[m + 1] >> 12) & 127)) ? (band[m + 1] & 4095) : zero;
    band[m] = hr | (hf << 12) | ((seg[m].y ? 1 : 0) << 24);
  }
  ok[2] = 1;
}

__global__ void mel_pack_kernel(float *packed, const float *W, const int4 *info, int n_mels, int nfreq) {
  const int m = blockIdx.x;
  if (m >= n_mels) return;
  const int4 in = info[m];
  for (int q = threadIdx.x; q < in.y; q += blockDim.x) packed[in.z + q] = W[(long long)m * nfreq + in.x + q];
}

// DCT-II ortho basis (MFCC.swift:79-88) in float64.
__global__ void build_dct_kernel(float *B, int n_mfcc, int n_mels) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_mfcc * n_mels) return;
  const int k = i / n_mels, n = i - k * n_mels;
  const long long num = ((long long)k * (2LL * n + 1)) % (4LL * n_mels);
  const double c = cospi((double)num / (2.0 * n_mels));
  const double s = (k == 0) ? sqrt(1.0 / n_mels) : sqrt(2.0 / n_mels);
  B[i] = (float)(c * s);
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
static inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t build_tables(DevTables &t, int sr, int n_fft, int win, int n_mels, float fmin,
                         float fmax, int n_mfcc_eff, int window_zero, cudaStream_t s) {
  cudaError_t e;
  const int nfreq = n_fft / 2 + 1;
  int log2n = 0;
  while ((1 << log2n) < n_fft) log2n++;
  t.n_fft = n_fft;
  t.n_mels = n_mels;
  t.n_mfcc = n_mfcc_eff;
#define MM_TRY(x) do { e = (x); if (e != cudaSuccess) return e; } while (0)
  MM_TRY(cudaMalloc(&t.window, sizeof(float) * (size_t)n_fft));
  build_window_kernel<<<blocks_for(n_fft, 256), 256, 0, s>>>(t.window, n_fft, win, window_zero);
  if (log2n >= 5) {
    const int log2m = log2n - 1;
    const int cnt = tw_count(log2m);
    MM_TRY(cudaMalloc(&t.tw_stage, sizeof(float2) * (size_t)(cnt > 0 ? cnt : 1)));
    const int ns_total = n_stages(log2m);
    for (int q = 1; q < ns_total; q++) {
      const int R = stage_radix(log2m, q), Ns = stage_ns(log2m, q);
      build_stage_tw_kernel<<<blocks_for((long long)(R - 1) * Ns, 256), 256, 0, s>>>(
          t.tw_stage + stage_tw_off(log2m, q), R, Ns);
    }
    const int m4 = n_fft / 4;
    MM_TRY(cudaMalloc(&t.tw_split, sizeof(float2) * (size_t)m4));
    build_roots_kernel<<<blocks_for(m4, 256), 256, 0, s>>>(t.tw_split, m4, n_fft);
  } else {
    MM_TRY(cudaMalloc(&t.tw_tiny, sizeof(float2) * (size_t)n_fft));
    build_roots_kernel<<<1, 32, 0, s>>>(t.tw_tiny, n_fft, n_fft);
  }
  if (n_mels > 0) {
    const long long cnt = (long long)n_mels * nfreq;
    int *d_nnz = nullptr;
    MM_TRY(cudaMalloc(&t.mel_w, sizeof(float) * (size_t)cnt));
    MM_TRY(cudaMalloc(&t.mel_info, sizeof(int4) * (size_t)n_mels));
    int *bin_seg = nullptr;
    MM_TRY(cudaMalloc(&d_nnz, 3 * sizeof(int)));
    MM_TRY(cudaMalloc(&t.mel_w2, sizeof(float2) * (size_t)nfreq));
    MM_TRY(cudaMalloc(&t.mel_seg, sizeof(int2) * (size_t)(n_mels + 1)));
    MM_TRY(cudaMalloc(&bin_seg, sizeof(int) * (size_t)nfreq));
    const int tpf = mel_lane_tpf(n_fft);
    if (tpf > 0) {
      MM_TRY(cudaMalloc(&t.mel_lw, sizeof(float2) * (size_t)(33 * tpf)));
      MM_TRY(cudaMalloc(&t.mel_lane, sizeof(int2) * (size_t)tpf));
      MM_TRY(cudaMalloc(&t.mel_band, sizeof(int) * (size_t)n_mels));
    }
    build_mel_kernel<<<blocks_for(cnt, 256), 256, 0, s>>>(t.mel_w, sr, n_fft, n_mels, (double)fmin,
                                                          (double)fmax);
    build_mel_info_kernel<<<blocks_for(n_mels, 128), 128, 0, s>>>(t.mel_info, t.mel_w, n_mels, nfreq);
    mel_offsets_kernel<<<1, 1, 0, s>>>(t.mel_info, n_mels, d_nnz);
    build_mel_bins_kernel<<<blocks_for(nfreq, 128), 128, 0, s>>>(t.mel_w2, bin_seg, t.mel_w, n_mels, nfreq);
    build_mel_seg_kernel<<<1, 1, 0, s>>>(t.mel_seg, bin_seg, t.mel_info, n_mels, nfreq, d_nnz);
    if (tpf > 0)
      build_mel_lane_kernel<<<1, 1, 0, s>>>(t.mel_lw, t.mel_lane, t.mel_band, t.mel_w2, bin_seg, t.mel_seg, n_mels,
                                            tpf, mel_lane_max_slots(tpf), d_nnz);
    int nnz_ok[3] = {0, 0, 0};
    e = cudaMemcpyAsync(nnz_ok, d_nnz, 3 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_nnz);
    cudaFree(bin_seg);
    if (e != cudaSuccess) return e;
    const int nnz = nnz_ok[0];
    t.mel_nnz = nnz;
    t.mel_seg_ok = nnz_ok[1];
    t.mel_lane_ok = tpf > 0 ? nnz_ok[2] : 0;
    MM_TRY(cudaMalloc(&t.mel_pw, sizeof(float) * (size_t)(nnz > 0 ? nnz : 1)));
    mel_pack_kernel<<<n_mels, 128, 0, s>>>(t.mel_pw, t.mel_w, t.mel_info, n_mels, nfreq);
  }
  if (n_mfcc_eff > 0 && n_mels > 0) {
    MM_TRY(cudaMalloc(&t.dct, sizeof(float) * (size_t)n_mfcc_eff * n_mels));
    build_dct_kernel<<<blocks_for((long long)n_mfcc_eff * n_mels, 256), 256, 0, s>>>(t.dct, n_mfcc_eff,
                                                                                      n_mels);
  }
#undef MM_TRY
  return cudaGetLastError();
}

// The dense filterbank [n_mels][n_fft/2+1] and its row info alone (the
// projection of a given spectrogram); n_fft need not be a power of two.
cudaError_t build_mel_dense(float *W, int4 *info, int sr, int n_fft, int n_mels, float fmin, float fmax,
                            cudaStream_t s) {
  const int nfreq = n_fft / 2 + 1;
  const long long cnt = (long long)n_mels * nfreq;
  if (cnt <= 0) return cudaSuccess;
  build_mel_kernel<<<blocks_for(cnt, 256), 256, 0, s>>>(W, sr, n_fft, n_mels, (double)fmin, (double)fmax);
  build_mel_info_kernel<<<blocks_for(n_mels, 128), 128, 0, s>>>(info, W, n_mels, nfreq);
  return cudaGetLastError();
}

// DCT-II ortho basis [n_out][n_rows] (float64-built, as the MFCC tables).
cudaError_t build_dct_basis_rows(float *B, int n_out, int n_rows, cudaStream_t s) {
  const long long cnt = (long long)n_out * n_rows;
  if (cnt <= 0) return cudaSuccess;
  build_dct_kernel<<<blocks_for(cnt, 256), 256, 0, s>>>(B, n_out, n_rows);
  return cudaGetLastError();
}

// Bump allocator over caller-provided device memory (256-byte aligned pieces).
namespace {
struct Carver {
  char *base;
  size_t cap, off;
  template <typename T>
  T *take(size_t count) {
    const size_t start = (off + 255) & ~size_t(255);
    const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    if (start + bytes > cap) return nullptr;
    off = start + bytes;
    return reinterpret_cast<T *>(base + start);
  }
};
}  // namespace

cudaError_t build_tables_at(DevTables &t, char *base, size_t cap, size_t *used, int sr, int n_fft,
                            int win, int n_mels, float fmin, float fmax, int n_mfcc_eff, int window_zero,
                            cudaStream_t s) {
  const int nfreq = n_fft / 2 + 1;
  int log2n = 0;
  while ((1 << log2n) < n_fft) log2n++;
  Carver c{base, cap, 0};
  t = DevTables();
  t.n_fft = n_fft;
  t.n_mels = n_mels;
  t.n_mfcc = n_mfcc_eff;
  if (!(t.window = c.take<float>(n_fft))) return cudaErrorMemoryAllocation;
  build_window_kernel<<<blocks_for(n_fft, 256), 256, 0, s>>>(t.window, n_fft, win, window_zero);
  if (log2n >= 5) {
    const int log2m = log2n - 1;
    if (!(t.tw_stage = c.take<float2>(tw_count(log2m)))) return cudaErrorMemoryAllocation;
    for (int q = 1; q < n_stages(log2m); q++) {
      const int R = stage_radix(log2m, q), Ns = stage_ns(log2m, q);
      build_stage_tw_kernel<<<blocks_for((long long)(R - 1) * Ns, 256), 256, 0, s>>>(
          t.tw_stage + stage_tw_off(log2m, q), R, Ns);
    }
    if (!(t.tw_split = c.take<float2>(n_fft / 4))) return cudaErrorMemoryAllocation;
    build_roots_kernel<<<blocks_for(n_fft / 4, 256), 256, 0, s>>>(t.tw_split, n_fft / 4, n_fft);
  } else {
    if (!(t.tw_tiny = c.take<float2>(n_fft))) return cudaErrorMemoryAllocation;
    build_roots_kernel<<<1, 32, 0, s>>>(t.tw_tiny, n_fft, n_fft);
  }
  if (n_mels > 0) {
    const long long cnt = (long long)n_mels * nfreq;
    int *d_nnz = nullptr;
    int *bin_seg = nullptr;
    const int tpf = mel_lane_tpf(n_fft);
    if (!(t.mel_w = c.take<float>(cnt)) || !(t.mel_info = c.take<int4>(n_mels)) || !(d_nnz = c.take<int>(3)) ||
        !(t.mel_w2 = c.take<float2>(nfreq)) || !(t.mel_seg = c.take<int2>(n_mels + 1)) ||
        !(bin_seg = c.take<int>(nfreq)))
      return cudaErrorMemoryAllocation;
    if (tpf > 0 && (!(t.mel_lw = c.take<float2>(33 * tpf)) || !(t.mel_lane = c.take<int2>(tpf)) ||
                    !(t.mel_band = c.take<int>(n_mels))))
      return cudaErrorMemoryAllocation;
    build_mel_kernel<<<blocks_for(cnt, 256), 256, 0, s>>>(t.mel_w, sr, n_fft, n_mels, (double)fmin,
                                                          (double)fmax);
    build_mel_info_kernel<<<blocks_for(n_mels, 128), 128, 0, s>>>(t.mel_info, t.mel_w, n_mels, nfreq);
    mel_offsets_kernel<<<1, 1, 0, s>>>(t.mel_info, n_mels, d_nnz);
    build_mel_bins_kernel<<<blocks_for(nfreq, 128), 128, 0, s>>>(t.mel_w2, bin_seg, t.mel_w, n_mels, nfreq);
    build_mel_seg_kernel<<<1, 1, 0, s>>>(t.mel_seg, bin_seg, t.mel_info, n_mels, nfreq, d_nnz);
    if (tpf > 0)
      build_mel_lane_kernel<<<1, 1, 0, s>>>(t.mel_lw, t.mel_lane, t.mel_band, t.mel_w2, bin_seg, t.mel_seg, n_mels,
                                            tpf, mel_lane_max_slots(tpf), d_nnz);
    int nnz_ok[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(nnz_ok, d_nnz, 3 * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    const int nnz = nnz_ok[0];
    t.mel_nnz = nnz;
    t.mel_seg_ok = nnz_ok[1];
    t.mel_lane_ok = tpf > 0 ? nnz_ok[2] : 0;
    if (!(t.mel_pw = c.take<float>(nnz))) return cudaErrorMemoryAllocation;
    mel_pack_kernel<<<n_mels, 128, 0, s>>>(t.mel_pw, t.mel_w, t.mel_info, n_mels, nfreq);
  }
  if (n_mfcc_eff > 0 && n_mels > 0) {
    if (!(t.dct = c.take<float>((long long)n_mfcc_eff * n_mels))) return cudaErrorMemoryAllocation;
    build_dct_kernel<<<blocks_for((long long)n_mfcc_eff * n_mels, 256), 256, 0, s>>>(t.dct, n_mfcc_eff,
                                                                                      n_mels);
  }
  if (used) *used = (c.off + 255) & ~size_t(255);
  return cudaGetLastError();
}

static int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Launch geometry of a persistent kernel, cached per (device, kernel, threads,
// dynamic shared memory), so that a launch costs no extra driver calls.  The
// kernel's shared-memory opt-in is one value per (device, kernel): it is only
// ever raised, so every size cached before stays launchable.
cudaError_t persistent_geometry(const void *kern, int threads, size_t smem, int *per_sm, int *sms) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void *, int, size_t>, std::pair<int, int>> cache;
  static std::map<std::pair<int, const void *>, size_t> opted_in;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const auto key = std::make_tuple(dev, kern, threads, smem);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) {
    *per_sm = it->second.first;
    *sms = it->second.second;
    return cudaSuccess;
  }
  size_t &opt = opted_in[std::make_pair(dev, kern)];
  if (smem > 48 * 1024 && smem > opt) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    opt = smem;
  }
  int p = 0, n = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, kern, threads, smem);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (p < 1) return cudaErrorInvalidConfiguration;
  cache[key] = {p, n};
  *per_sm = p;
  *sms = n;
  return cudaSuccess;
}

template <bool TINY, typename K>
static cudaError_t launch_persistent(K kern, int threads, size_t smem, int tiles, int grid_limit,
                                     size_t *configured, const FrontArgs &a, cudaStream_t s,
                                     int *launched, int n_fft) {
  (void)configured;
  int per_sm = 1, sms = 148;
  cudaError_t e = persistent_geometry(reinterpret_cast<const void *>(kern), threads, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = (long long)sms * per_sm;
  if (grid_limit > 0 && grid > grid_limit) grid = grid_limit;
  if (grid > tiles) grid = tiles;
  if (grid < 1) return cudaSuccess;
  if constexpr (TINY) kern<<<(unsigned)grid, threads, smem, s>>>(a, n_fft);
  else kern<<<(unsigned)grid, threads, smem, s>>>(a);
  if (launched) *launched = (int)grid;
  return cudaGetLastError();
}

template <int LOG2N, int V, int MODE, int PW>
static cudaError_t launch_fft_t(const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched) {
  using C = Cfg<LOG2N, V>;
  const size_t smem = fixed_smem_bytes<LOG2N, C::F>() +
                      (mode_has_mel(MODE) ? mel_smem_bytes(a.n_mels, a.mel_nnz) : 0);
  static size_t configured = 0;
  return launch_persistent<false>(frontend_kernel<LOG2N, V, MODE, PW>, C::THREADS, smem, a.total_tiles,
                                  grid_limit, &configured, a, s, launched, 1 << LOG2N);
}

template <int LOG2N, int MODE, int PW>
static cudaError_t launch_size(int v, const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched) {
  if constexpr (tunable(LOG2N, MODE, PW)) {
    if (v == 1) return launch_fft_t<LOG2N, 1, MODE, PW>(a, grid_limit, s, launched);
    if (v == 2) return launch_fft_t<LOG2N, 2, MODE, PW>(a, grid_limit, s, launched);
  }
  return launch_fft_t<LOG2N, 0, MODE, PW>(a, grid_limit, s, launched);
}

template <int MODE, int PW>
static cudaError_t launch_mode(int log2n, int v, const FrontArgs &a, int grid_limit, cudaStream_t s,
                               int *launched) {
  switch (log2n) {
    case 5: return launch_size<5, MODE, PW>(v, a, grid_limit, s, launched);
    case 6: return launch_size<6, MODE, PW>(v, a, grid_limit, s, launched);
    case 7: return launch_size<7, MODE, PW>(v, a, grid_limit, s, launched);
    case 8: return launch_size<8, MODE, PW>(v, a, grid_limit, s, launched);
    case 9: return launch_size<9, MODE, PW>(v, a, grid_limit, s, launched);
    case 10: return launch_size<10, MODE, PW>(v, a, grid_limit, s, launched);
    case 11: return launch_size<11, MODE, PW>(v, a, grid_limit, s, launched);
    case 12: return launch_size<12, MODE, PW>(v, a, grid_limit, s, launched);
    case 13: return launch_size<13, MODE, PW>(v, a, grid_limit, s, launched);
    case 14: return launch_size<14, MODE, PW>(v, a, grid_limit, s, launched);
    case 15: return launch_size<15, MODE, PW>(v, a, grid_limit, s, launched);
    default: break;
  }
  if (log2n < 0 || log2n > 4) return cudaErrorInvalidValue;
  const size_t smem = mode_has_mel(MODE) ? mel_smem_bytes(a.n_mels, a.mel_nnz) : 0;
  static size_t configured = 0;
  return launch_persistent<true>(frontend_tiny_kernel<MODE, PW>, 128, smem, a.total_tiles, grid_limit,
                                 &configured, a, s, launched, 1 << log2n);
}

cudaError_t launch_frontend(int log2n, int mode, int variant, const FrontArgs &a, int grid_limit,
                            cudaStream_t s, int *launched) {
  if (launched) *launched = 0;
  if (a.total_tiles <= 0) return cudaSuccess;
  const int pw = (a.power == 2.0f) ? 0 : (a.power == 1.0f ? 1 : 2);
  switch (mode) {
    case MODE_SPECTRUM:
      if (pw == 0) return launch_mode<MODE_SPECTRUM, 0>(log2n, variant, a, grid_limit, s, launched);
      if (pw == 1) return launch_mode<MODE_SPECTRUM, 1>(log2n, variant, a, grid_limit, s, launched);
      return launch_mode<MODE_SPECTRUM, 2>(log2n, variant, a, grid_limit, s, launched);
    case MODE_MEL:
      if (pw == 0) return launch_mode<MODE_MEL, 0>(log2n, variant, a, grid_limit, s, launched);
      if (pw == 1) return launch_mode<MODE_MEL, 1>(log2n, variant, a, grid_limit, s, launched);
      return launch_mode<MODE_MEL, 2>(log2n, variant, a, grid_limit, s, launched);
    case MODE_COMPLEX: return launch_mode<MODE_COMPLEX, 0>(log2n, variant, a, grid_limit, s, launched);
    case MODE_MELDB:
      if (pw != 0) return cudaErrorInvalidValue;
      if (variant == kTcVariant && log2n == 11) return launch_frontend_tc(a, grid_limit, s, launched);
      if (variant == kWarpVariant && warp_frames_per_tile(log2n) > 0)
        return launch_frontend_warp(log2n, a, grid_limit, s, launched);
      return launch_mode<MODE_MELDB, 0>(log2n, variant, a, grid_limit, s, launched);
    default: return cudaErrorInvalidValue;
  }
}

// The same product with whole rows: the basis [n_mfcc][n_mels] is staged once
// per CTA and each 64-frame tile is loaded over all bands at once (one
// barrier pair per tile).  Row stride n_mels + pad with stride % 32 == 4 keeps
// the float4 row reads of the 64 frames conflict-free.  n_mels % 4 == 0,
// n_mels <= 256, n_mfcc <= 32.
__host__ __device__ inline int dct_row_stride(int n_mels) { return n_mels + ((36 - (n_mels & 31)) & 31); }

template <int KQ>
__global__ void __launch_bounds__(256, 3) dct_rows_kernel(DctArgs a) {
  extern __shared__ __align__(16) float dsm[];
  const int nm = a.n_mels, stride = dct_row_stride(nm), n4 = nm / 4;
  float *bas = dsm;                      // [4*KQ][nm]
  float *tile = dsm + 4 * KQ * nm;       // [64][stride]
  const int tid = threadIdx.x;
  const int fr = tid & (kDctTile - 1), kg = tid / kDctTile;
  for (int i = tid; i < 4 * KQ * nm; i += 256) {
    const int k = i / nm;
    bas[i] = k < a.n_mfcc ? __ldg(a.basis + i) : 0.0f;
  }
  const float4 *brow = reinterpret_cast<const float4 *>(bas + kg * KQ * nm);
  const float4 *trow = reinterpret_cast<const float4 *>(tile + fr * stride);
  for (int ti = blockIdx.x; ti < a.total_tiles; ti += gridDim.x) {
    const int c = __ldg(a.tile_clip + ti);
    const ClipDesc cd = load_clip(a.clips + c);
    const int tf = __ldg(a.tile_first + ti);
    const int nt = min(kDctTile, cd.n_frames - tf);
    const bool floor_on = a.top_db > 0.0f;
    const float thr = floor_on ? dec_f(__ldg(a.clip_max + c)) - a.top_db : 0.0f;
    const float4 *src = reinterpret_cast<const float4 *>(a.mel_db + (cd.frame_off + tf) * (long long)nm);
    __syncthreads();  // the previous tile's reads are done
    for (int i = tid; i < kDctTile * n4; i += 256) {
      const int r = i / n4, c4 = i - r * n4;
      float4 v = r < nt ? __ldg(src + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      if (floor_on && r < nt) {
        v.x = vthr(v.x, thr);
        v.y = vthr(v.y, thr);
        v.z = vthr(v.z, thr);
        v.w = vthr(v.w, thr);
      }
      *reinterpret_cast<float4 *>(tile + r * stride + 4 * c4) = v;
    }
    __syncthreads();
    float acc[KQ];
#pragma unroll
    for (int q = 0; q < KQ; q++) acc[q] = 0.0f;
#pragma unroll 2
    for (int j = 0; j < n4; j++) {
      const float4 d = trow[j];
#pragma unroll
      for (int q = 0; q < KQ; q++) {
        const float4 b = brow[q * n4 + j];
        acc[q] = fmaf(b.x, d.x, acc[q]);
        acc[q] = fmaf(b.y, d.y, acc[q]);
        acc[q] = fmaf(b.z, d.z, acc[q]);
        acc[q] = fmaf(b.w, d.w, acc[q]);
      }
    }
    if (fr < nt) {
      const long long T = cd.n_frames;
#pragma unroll
      for (int q = 0; q < KQ; q++) {
        const int k = kg * KQ + q;
        if (k < a.n_mfcc) a.out[cd.out_off + (long long)k * T + tf + fr] = acc[q];
      }
    }
  }
}

// The same whole-row product, software-pipelined (n_mels <= 128): while a
// tile is multiplied out of shared memory, each thread already holds its part
// of the next tile's rows in registers (at most 8 float4: 64 frames x n_mels/4
// float4 over 256 threads), so the HBM latency of the next tile overlaps the
// arithmetic of this one.  The rows are floored at the clip's threshold on the
// way into shared memory, as in dct_rows_kernel.
constexpr int kDctPipeVec = 8;  // float4 per thread and tile (n_mels <= 128)

struct DctTileMeta {
  long long out_off, T;
  const float4 *src;
  int tf, nt;
  float thr;
};

__device__ __forceinline__ DctTileMeta dct_tile_meta(const DctArgs &a, int ti) {
  DctTileMeta m;
  const int c = __ldg(a.tile_clip + ti);
  const ClipDesc cd = load_clip(a.clips + c);
  m.tf = __ldg(a.tile_first + ti);
  m.nt = min(kDctTile, cd.n_frames - m.tf);
  m.thr = a.top_db > 0.0f ? dec_f(__ldg(a.clip_max + c)) - a.top_db : -INFINITY;
  m.src = reinterpret_cast<const float4 *>(a.mel_db + (cd.frame_off + m.tf) * (long long)a.n_mels);
  m.out_off = cd.out_off;
  m.T = cd.n_frames;
  return m;
}

// NM > 0: n_mels fixed at compile time (the product unrolls with immediate
// shared-memory offsets); NM == 0: any n_mels <= 128.
template <int KQ, int NM>
__global__ void __launch_bounds__(256, 2) dct_pipe_kernel(DctArgs a) {
  extern __shared__ __align__(16) float dsm[];
  const int nm = NM > 0 ? NM : a.n_mels, stride = dct_row_stride(nm), n4 = nm / 4, cnt = kDctTile * n4;
  float *bas = dsm;                 // [4*KQ][nm]
  float *tile = dsm + 4 * KQ * nm;  // [64][stride]
  const int tid = threadIdx.x;
  const int fr = tid & (kDctTile - 1), kg = tid / kDctTile;
  for (int i = tid; i < 4 * KQ * nm; i += 256) {
    const int k = i / nm;
    bas[i] = k < a.n_mfcc ? __ldg(a.basis + i) : 0.0f;
  }
  const float4 *brow = reinterpret_cast<const float4 *>(bas + kg * KQ * nm);
  const float4 *trow = reinterpret_cast<const float4 *>(tile + fr * stride);
  int ti = blockIdx.x;
  if (ti >= a.total_tiles) return;
  float4 pre[kDctPipeVec];
  DctTileMeta cur = dct_tile_meta(a, ti);
#pragma unroll
  for (int v = 0; v < kDctPipeVec; v++) {
    const int i = tid + 256 * v;
    pre[v] = (i < cnt && i / n4 < cur.nt) ? __ldg(cur.src + i) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (; ti < a.total_tiles; ti += gridDim.x) {
    __syncthreads();  // every thread is done with the previous tile in shared memory
#pragma unroll
    for (int v = 0; v < kDctPipeVec; v++) {
      const int i = tid + 256 * v;
      if (i < cnt) {
        const int r = i / n4, c4 = i - r * n4;
        float4 x = pre[v];
        if (r < cur.nt) {
          x.x = vthr(x.x, cur.thr);
          x.y = vthr(x.y, cur.thr);
          x.z = vthr(x.z, cur.thr);
          x.w = vthr(x.w, cur.thr);
        }
        *reinterpret_cast<float4 *>(tile + r * stride + 4 * c4) = x;
      }
    }
    __syncthreads();
    // next tile's rows into registers while this one is multiplied
    const int nti = ti + gridDim.x;
    DctTileMeta nxt = cur;
    if (nti < a.total_tiles) {
      nxt = dct_tile_meta(a, nti);
#pragma unroll
      for (int v = 0; v < kDctPipeVec; v++) {
        const int i = tid + 256 * v;
        pre[v] = (i < cnt && i / n4 < nxt.nt) ? __ldg(nxt.src + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    float acc[KQ];
#pragma unroll
    for (int q = 0; q < KQ; q++) acc[q] = 0.0f;
    if constexpr (NM > 0) {
#pragma unroll
      for (int j = 0; j < NM / 4; j++) {
        const float4 d = trow[j];
#pragma unroll
        for (int q = 0; q < KQ; q++) {
          const float4 b = brow[q * (NM / 4) + j];
          acc[q] = fmaf(b.x, d.x, acc[q]);
          acc[q] = fmaf(b.y, d.y, acc[q]);
          acc[q] = fmaf(b.z, d.z, acc[q]);
          acc[q] = fmaf(b.w, d.w, acc[q]);
        }
      }
    } else {
#pragma unroll 2
      for (int j = 0; j < n4; j++) {
        const float4 d = trow[j];
#pragma unroll
        for (int q = 0; q < KQ; q++) {
          const float4 b = brow[q * n4 + j];
          acc[q] = fmaf(b.x, d.x, acc[q]);
          acc[q] = fmaf(b.y, d.y, acc[q]);
          acc[q] = fmaf(b.z, d.z, acc[q]);
          acc[q] = fmaf(b.w, d.w, acc[q]);
        }
      }
    }
    if (fr < cur.nt) {
#pragma unroll
      for (int q = 0; q < KQ; q++) {
        const int k = kg * KQ + q;
        if (k < a.n_mfcc) a.out[cur.out_off + (long long)k * cur.T + cur.tf + fr] = acc[q];
      }
    }
    cur = nxt;
  }
}

// NM bands (64, 80 or 128: a multiple of 16, so a half row is an even number
// of float4 chunks): the DCT-II basis is symmetric in n for even k and antisymmetric
// for odd k (cos(pi k (2(N-1-n)+1) / 2N) = (-1)^k cos(pi k (2n+1) / 2N)), so
// with e_n = x_n + x_{N-1-n} and o_n = x_n - x_{N-1-n} (n < N/2) the even
// coefficients are sum_n B[k][n] e_n and the odd ones sum_n B[k][n] o_n: half
// the products and half the basis reads.
// Coefficient groups (one per warp): kg 0, 1 take even k = 2 (KQ kg + q),
// kg 2, 3 odd k = 2 (KQ (kg - 2) + q) + 1, so KQ = ceil(ceil(n_mfcc / 2) / 2).
// Per tile of 64 frames (the summation order of the other DCT kernels: float4
// chunk by chunk, x, y, z, w):
// - a tile's rows are copied straight into shared memory by cp.async (no
//   registers in flight), two tile buffers, the next tile's copies issued
//   before this one is folded;
// - the floor and the even/odd fold run in place in shared memory: with C4 =
//   NM / 4 chunks a row and H4 = C4 / 2, a thread takes float4 chunks j,
//   H4 - 1 - j of a row and their mirrors C4 - 1 - j, H4 + j, reads all four,
//   then writes e over chunks j, H4 - 1 - j and o over H4 + j, C4 - 1 - j
//   (the row becomes [e | o]);
// - 128 threads, each two frames (lane, lane + 32) x KQ coefficients of its
//   warp's group, so every basis read from shared memory feeds two frames.
// floats per staged row: NM + 4 mod 32 (16-byte aligned; a warp's 32 row reads conflict-free)
__host__ __device__ constexpr int dct2_stride(int nm) { return nm + ((36 - (nm & 31)) & 31); }
// Tile buffers in the copy ring: two (3 CTAs per SM) measured 0.0618 ms per
// bench step against 0.0677 ms for three (2 CTAs per SM).
constexpr int kDctFoldStages = 2;

template <int KQ, int S, int NM>
__global__ void __launch_bounds__(128, S == 2 ? 3 : 2) dct_fold2_kernel(DctArgs a) {
  static_assert(NM % 16 == 0 && NM <= 128, "a half row must be an even number of float4 chunks");
  constexpr int H = NM / 2, H4 = H / 4, C4 = NM / 4, TS = dct2_stride(NM);
  extern __shared__ __align__(16) float dsm[];
  float *buf0 = dsm;                     // [kDctTile][TS] x S
  float *bas = dsm + S * kDctTile * TS;  // [4*KQ][H]
  const int tid = threadIdx.x, lane = tid & 31, kg = tid >> 5;
  auto coef = [](int g, int q) { return g < 2 ? 2 * (KQ * g + q) : 2 * (KQ * (g - 2) + q) + 1; };
  for (int i = tid; i < 4 * KQ * H; i += 128) {
    const int row = i / H, n = i - row * H;
    const int k = coef(row / KQ, row % KQ);
    bas[i] = k < a.n_mfcc ? __ldg(a.basis + (long long)k * NM + n) : 0.0f;
  }
  int ti = blockIdx.x;
  if (ti >= a.total_tiles) return;
  // A tile's meta takes three dependent loads (tile -> clip -> descriptor and
  // maximum); they are spread over the tile S ahead of the one multiplied:
  // its tile words at the top, its clip's words after the fold, the meta put
  // together after the product, so no warp waits on a chain of loads.
  auto finish_meta = [&](int c, int tf, const ClipDesc &cd, unsigned cm) {
    DctTileMeta m;
    m.tf = tf;
    m.nt = min(kDctTile, cd.n_frames - tf);
    m.thr = a.top_db > 0.0f ? dec_f(cm) - a.top_db : -INFINITY;
    m.src = reinterpret_cast<const float4 *>(a.mel_db + (cd.frame_off + tf) * (long long)NM);
    m.out_off = cd.out_off;
    m.T = cd.n_frames;
    return m;
  };
  // rows r < nt of tile m into buffer b: chunk i = tid + 128 u is row i / C4, float4 i % C4
  auto issue = [&](const DctTileMeta &m, float *b) {
    static_assert(kDctTile * C4 % 128 == 0, "whole copy rounds");
#pragma unroll
    for (int u = 0; u < kDctTile * C4 / 128; u++) {
      const int i = tid + 128 * u, r = i / C4, c4 = i - r * C4;
      if (r < m.nt) cp_async16(b + r * TS + 4 * c4, m.src + r * C4 + c4);
    }
    cp_async_commit();
  };
  const int G = gridDim.x;
  // m[0]: this tile; m[s]: the tile s ahead (copies issued for s < S - 1)
  DctTileMeta m[S];
  m[0] = dct_tile_meta(a, ti);
  issue(m[0], buf0);
#pragma unroll
  for (int q = 1; q < S; q++) {
    m[q] = m[q - 1];
    if (ti + q * G < a.total_tiles) {
      m[q] = dct_tile_meta(a, ti + q * G);
      if (q < S - 1) issue(m[q], buf0 + q * kDctTile * TS);
    }
  }
  const float4 *brow = reinterpret_cast<const float4 *>(bas + kg * KQ * H);
  for (int k = 0; ti < a.total_tiles; ti += G, k++) {
    const DctTileMeta &cur = m[0];
    float *b = buf0 + (k % S) * kDctTile * TS;
    // copies of the tile S - 1 ahead into the buffer released at the end of
    // tile k - 1, then wait for this tile's (tiles after it stay in flight)
    const int ahead = min(S - 1, (a.total_tiles - 1 - ti) / G);
    if (ahead == S - 1) issue(m[S - 1], buf0 + ((k + S - 1) % S) * kDctTile * TS);
    if (S == 3 && ahead >= 2) cp_async_wait<2>();
    else if (ahead >= 1) cp_async_wait<1>();
    else cp_async_wait<0>();
    // tile words of the tile S ahead
    const int t2 = ti + S * G;
    const bool has2 = t2 < a.total_tiles;
    int c2 = 0, f2 = 0;
    if (has2) {
      c2 = __ldg(a.tile_clip + t2);
      f2 = __ldg(a.tile_first + t2);
    }
    __syncthreads();  // every thread's copies of this tile have landed
    // floor + fold in place: unit i is row i / (H4 / 2), chunk pair j = i % (H4 / 2)
#pragma unroll
    for (int i = tid; i < kDctTile * (H4 / 2); i += 128) {
      const int r = i / (H4 / 2), j = i - r * (H4 / 2);
      if (r < cur.nt) {
        float4 *row = reinterpret_cast<float4 *>(b + r * TS);
        float4 A = row[j], Am = row[C4 - 1 - j], B = row[H4 - 1 - j], Bm = row[H4 + j];
        const float t = cur.thr;
        A = make_float4(vthr(A.x, t), vthr(A.y, t), vthr(A.z, t), vthr(A.w, t));
        Am = make_float4(vthr(Am.x, t), vthr(Am.y, t), vthr(Am.z, t), vthr(Am.w, t));
        B = make_float4(vthr(B.x, t), vthr(B.y, t), vthr(B.z, t), vthr(B.w, t));
        Bm = make_float4(vthr(Bm.x, t), vthr(Bm.y, t), vthr(Bm.z, t), vthr(Bm.w, t));
        row[j] = make_float4(A.x + Am.w, A.y + Am.z, A.z + Am.y, A.w + Am.x);
        row[H4 + j] = make_float4(A.x - Am.w, A.y - Am.z, A.z - Am.y, A.w - Am.x);
        row[H4 - 1 - j] = make_float4(B.x + Bm.w, B.y + Bm.z, B.z + Bm.y, B.w + Bm.x);
        row[C4 - 1 - j] = make_float4(B.x - Bm.w, B.y - Bm.z, B.z - Bm.y, B.w - Bm.x);
      }
    }
    // its clip's words
    ClipDesc cd2{};
    unsigned cm2 = 0;
    if (has2) {
      cd2 = load_clip(a.clips + c2);
      cm2 = __ldg(a.clip_max + c2);
    }
    __syncthreads();
    const float4 *t0 = reinterpret_cast<const float4 *>(b + lane * TS + (kg < 2 ? 0 : H));
    const float4 *t1 = t0 + 32 * TS / 4;
    float acc0[KQ], acc1[KQ];
#pragma unroll
    for (int q = 0; q < KQ; q++) acc0[q] = acc1[q] = 0.0f;
#pragma unroll
    for (int j = 0; j < H4; j++) {
      const float4 d0 = t0[j], d1 = t1[j];
#pragma unroll
      for (int q = 0; q < KQ; q++) {
        const float4 w = brow[q * H4 + j];
        acc0[q] = fmaf(w.x, d0.x, acc0[q]);
        acc0[q] = fmaf(w.y, d0.y, acc0[q]);
        acc0[q] = fmaf(w.z, d0.z, acc0[q]);
        acc0[q] = fmaf(w.w, d0.w, acc0[q]);
        acc1[q] = fmaf(w.x, d1.x, acc1[q]);
        acc1[q] = fmaf(w.y, d1.y, acc1[q]);
        acc1[q] = fmaf(w.z, d1.z, acc1[q]);
        acc1[q] = fmaf(w.w, d1.w, acc1[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < KQ; q++) {
      const int kk = coef(kg, q);
      if (kk < a.n_mfcc) {
        float *o = a.out + cur.out_off + (long long)kk * cur.T + cur.tf;
        if (lane < cur.nt) o[lane] = acc0[q];
        if (lane + 32 < cur.nt) o[lane + 32] = acc1[q];
      }
    }
    __syncthreads();  // this tile's buffer is free for the copies of tile k + S
#pragma unroll
    for (int q = 0; q < S - 1; q++) m[q] = m[q + 1];
    if (has2) m[S - 1] = finish_meta(c2, f2, cd2, cm2);
  }
}

template <int KQ, int S, int NM>
static cudaError_t launch_dct_fold2_s(const DctArgs &a, cudaStream_t s) {
  const size_t smem = sizeof(float) * ((size_t)S * kDctTile * dct2_stride(NM) + (size_t)4 * KQ * (NM / 2));
  int per_sm = 1, sms = 148;
  cudaError_t e =
      persistent_geometry(reinterpret_cast<const void *>(dct_fold2_kernel<KQ, S, NM>), 128, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = (long long)sms * per_sm;
  if (grid > a.total_tiles) grid = a.total_tiles;
  dct_fold2_kernel<KQ, S, NM><<<(unsigned)grid, 128, smem, s>>>(a);
  return cudaGetLastError();
}

// n_mels 64, 80 or 128 (the bands of the default, speech and mixed-batch front ends)
template <int KQ>
static cudaError_t launch_dct_fold2_t(const DctArgs &a, cudaStream_t s) {
  switch (a.n_mels) {
    case 64: return launch_dct_fold2_s<KQ, kDctFoldStages, 64>(a, s);
    case 80: return launch_dct_fold2_s<KQ, kDctFoldStages, 80>(a, s);
    default: return launch_dct_fold2_s<KQ, kDctFoldStages, 128>(a, s);
  }
}

template <int KQ>
static cudaError_t launch_dct_pipe_t(const DctArgs &a, cudaStream_t s) {
  const size_t smem = sizeof(float) * ((size_t)4 * KQ * a.n_mels + (size_t)kDctTile * dct_row_stride(a.n_mels));
  auto kern = a.n_mels == 128 ? dct_pipe_kernel<KQ, 128> : dct_pipe_kernel<KQ, 0>;
  int per_sm = 1, sms = 148;
  cudaError_t e = persistent_geometry(reinterpret_cast<const void *>(kern), 256, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = (long long)sms * per_sm;
  if (grid > a.total_tiles) grid = a.total_tiles;
  kern<<<(unsigned)grid, 256, smem, s>>>(a);
  return cudaGetLastError();
}

template <int KQ>
static cudaError_t launch_dct_rows_t(const DctArgs &a, cudaStream_t s) {
  const size_t smem = sizeof(float) * ((size_t)4 * KQ * a.n_mels + (size_t)kDctTile * dct_row_stride(a.n_mels));
  int per_sm = 1, sms = 148;
  cudaError_t e = persistent_geometry(reinterpret_cast<const void *>(dct_rows_kernel<KQ>), 256, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = (long long)sms * per_sm;
  if (grid > a.total_tiles) grid = a.total_tiles;
  dct_rows_kernel<KQ><<<(unsigned)grid, 256, smem, s>>>(a);
  return cudaGetLastError();
}

template <int KQ>
static cudaError_t launch_dct_t(const DctArgs &a, cudaStream_t s) {
  static int sms = 0;
  if (sms == 0) sms = sm_count();
  long long grid = (long long)sms * 4;
  if (grid > a.total_tiles) grid = a.total_tiles;
  dct_kernel<KQ><<<(unsigned)grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_dct(const DctArgs &a, cudaStream_t s) {
  if (a.total_tiles <= 0 || a.n_mfcc <= 0) return cudaSuccess;
  // 4 coefficient groups x KQ accumulators cover min(n_mfcc, 32) coefficients per pass
  const int kq = (std::min(a.n_mfcc, kDctKC) + 3) / 4;
  if (a.n_mfcc <= kDctKC && (a.n_mels == 128 || a.n_mels == 80 || a.n_mels == 64)) {
    switch ((a.n_mfcc + 3) / 4) {  // ceil(ceil(n_mfcc / 2) / 2)
      case 1: return launch_dct_fold2_t<1>(a, s);
      case 2: return launch_dct_fold2_t<2>(a, s);
      case 3: return launch_dct_fold2_t<3>(a, s);
      case 4: return launch_dct_fold2_t<4>(a, s);
      case 5: return launch_dct_fold2_t<5>(a, s);
      case 6: return launch_dct_fold2_t<6>(a, s);
      case 7: return launch_dct_fold2_t<7>(a, s);
      default: return launch_dct_fold2_t<8>(a, s);
    }
  }
  if (a.n_mfcc <= kDctKC && a.n_mels % 4 == 0 && a.n_mels <= 4 * kDctPipeVec * 256 / kDctTile) {
    switch (kq) {
      case 1: return launch_dct_pipe_t<1>(a, s);
      case 2: return launch_dct_pipe_t<2>(a, s);
      case 3: return launch_dct_pipe_t<3>(a, s);
      case 4: return launch_dct_pipe_t<4>(a, s);
      case 5: return launch_dct_pipe_t<5>(a, s);
      case 6: return launch_dct_pipe_t<6>(a, s);
      case 7: return launch_dct_pipe_t<7>(a, s);
      default: return launch_dct_pipe_t<8>(a, s);
    }
  }
  if (a.n_mfcc <= kDctKC && a.n_mels % 4 == 0 && a.n_mels <= 256) {
    switch (kq) {
      case 1: return launch_dct_rows_t<1>(a, s);
      case 2: return launch_dct_rows_t<2>(a, s);
      case 3: return launch_dct_rows_t<3>(a, s);
      case 4: return launch_dct_rows_t<4>(a, s);
      case 5: return launch_dct_rows_t<5>(a, s);
      case 6: return launch_dct_rows_t<6>(a, s);
      case 7: return launch_dct_rows_t<7>(a, s);
      default: return launch_dct_rows_t<8>(a, s);
    }
  }
  switch (kq) {
    case 1: return launch_dct_t<1>(a, s);
    case 2: return launch_dct_t<2>(a, s);
    case 3: return launch_dct_t<3>(a, s);
    case 4: return launch_dct_t<4>(a, s);
    case 5: return launch_dct_t<5>(a, s);
    case 6: return launch_dct_t<6>(a, s);
    case 7: return launch_dct_t<7>(a, s);
    default: return launch_dct_t<8>(a, s);
  }
}

cudaError_t launch_fill_u32(unsigned *p, unsigned v, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  long long g = (n + 255) / 256;
  if (g > 4096) g = 4096;
  fill_u32_kernel<<<(unsigned)g, 256, 0, s>>>(p, v, n);
  return cudaGetLastError();
}

cudaError_t launch_fill_pattern(float *p, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  long long g = (n + 255) / 256;
  if (g > 4096) g = 4096;
  fill_pattern_kernel<<<(unsigned)g, 256, 0, s>>>(p, n);
  return cudaGetLastError();
}

cudaError_t launch_db(const float *x, float *y, long long n, float mult, float amin, float ref,
                      float top_db, unsigned *slot, cudaStream_t s, unsigned *ref_slot) {
  if (n <= 0) return cudaSuccess;
  cudaError_t e = launch_fill_u32(slot, encode_max_init(), 1, s);
  if (e != cudaSuccess) return e;
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  if (ref_slot) {
    if ((e = launch_fill_u32(ref_slot, encode_max_init(), 1, s)) != cudaSuccess) return e;
    if ((e = launch_fill_u32(ref_slot + 1, 0u, 1, s)) != cudaSuccess) return e;
    db_ref_kernel<<<(unsigned)g, 256, 0, s>>>(x, n, ref_slot);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  db_pass1_kernel<<<(unsigned)g, 256, 0, s>>>(x, y, n, mult, amin, ref, ref_slot, slot);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (top_db > 0.0f) {
    db_pass2_kernel<<<(unsigned)g, 256, 0, s>>>(y, n, top_db, slot);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace mm
