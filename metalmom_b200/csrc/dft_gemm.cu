// DFT as a GEMM on the 5th-generation tensor cores (tcgen05, sm_100a): the
// precision-comparison form of the front end (n_fft 256..1024, MFCC path).
//
// The reference transforms each frame with Accelerate's radix-2 real FFT
// (STFT.swift:287-310); here the same spectrum is one matrix product per tile
// of 128 frames:
//
//   X[t][c] = sum_j A[t][j] B[c][j]
//   A[t][j] = x[t*hop - pad + k0 + j]                 (frame samples)
//   B[2k][j] = w[k0+j] cos(2 pi (k0+j) k / N),  B[2k+1][j] = -w[k0+j] sin(...)
//
// j runs over the window's support only (k0.. k0+kw, kw a multiple of 64),
// so the window multiply lives in B.  A and B are split into bf16 parts
// (v = hi + lo); the BF16x3 form accumulates hi*hi + hi*lo + lo*hi in one
// float32 TMEM accumulator, the plain BF16 form hi*hi only.
//
// Per CTA (128 threads, one frame per thread = one TMEM lane), per N tile of
// at most 256 columns, per K chunk of 64: the threads write the A chunk (from
// the signal) and the B chunk (a pre-swizzled image) into shared memory in
// the K-major 128-byte-swizzle layout, thread 0 issues the tcgen05.mma
// instructions and commits them to an mbarrier.  After the last chunk each
// warp reads its 32 lanes of the accumulator (tcgen05.ld), forms |X|^2, and
// folds the bins into the mel bands with the per-bin split of the filterbank
// (band m = R[m] + F[m+1]); the log-mel row and the clip maximum are written as
// by the FFT kernels, and the same DCT kernel follows.
//
// Every wait is bounded: a wait that runs out sets the error word and the
// CTA stops, releases its tensor memory and returns.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "frame_common.cuh"
#include "kernels.h"

namespace mm {

constexpr int kDftM = 128;   // frames per tile = TMEM lanes
constexpr int kDftKC = 64;   // K per chunk: one 128-byte swizzle row of bf16
constexpr int kDftThreads = 256;  // 8 warps: two per TMEM lane quarter
constexpr int kDftTmemCols = 256;
constexpr size_t kDftMinSmem = 80 * 1024;  // at most two CTAs per SM: 2 x 256 TMEM columns

DftShape dft_shape(int n_fft, int win) {
  DftShape s{};
  s.n_fft = n_fft;
  s.nbins = n_fft / 2 + 1;
  const int ncols = 2 * s.nbins;
  s.ntiles = (ncols + 255) / 256;
  s.tile_cols = 16 * ((ncols + 16 * s.ntiles - 1) / (16 * s.ntiles));
  const int w = (win > 0 && win < n_fft) ? win : n_fft;
  const int pad_w = (n_fft - w) / 2;
  s.kw = (w + kDftKC - 1) / kDftKC * kDftKC;
  for (;;) {
    s.k0 = std::min(pad_w & ~3, n_fft - s.kw);
    if (s.k0 + s.kw >= pad_w + w || s.kw >= n_fft) break;
    s.kw += kDftKC;
  }
  if (s.kw > n_fft) s.kw = n_fft;
  s.k0 = std::max(0, std::min(s.k0, n_fft - s.kw));
  s.kchunks = s.kw / kDftKC;
  return s;
}

bool dft_supported(int n_fft, int win) { return n_fft >= 256 && n_fft <= 1024 && win > 0 && win <= n_fft; }

size_t dft_basis_bytes(const DftShape &s) {
  return (size_t)s.ntiles * s.kchunks * 2 * (size_t)s.tile_cols * 128;
}

// Byte offset of element (row r, k) in a K-major tile with 128-byte rows and
// the 128-byte swizzle (16-byte chunk index XOR row % 8).
__host__ __device__ __forceinline__ uint32_t sw128(int r, int k) {
  return (uint32_t)r * 128u + ((uint32_t)(((k >> 3) ^ (r & 7))) << 4) + (uint32_t)(k & 7) * 2u;
}

// B image: [tile][chunk][part hi/lo][tile_cols rows x 128 bytes], values in
// float64 (window and twiddle), split into bf16 hi + lo.
__global__ void build_dft_basis_kernel(__nv_bfloat16 *img, DftShape s, int win, int window_zero) {
  const long long total = (long long)s.ntiles * s.kchunks * s.tile_cols * kDftKC;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int j = (int)(i % kDftKC);
  long long q = i / kDftKC;
  const int r = (int)(q % s.tile_cols);
  q /= s.tile_cols;
  const int kc = (int)(q % s.kchunks);
  const int nt = (int)(q / s.kchunks);
  const int col = nt * s.tile_cols + r;
  const int bin = col >> 1, part = col & 1;
  const int n = s.k0 + kc * kDftKC + j;
  double v = 0.0;
  if (bin < s.nbins && n < s.n_fft && !window_zero) {
    const int w_len = (win > 0 && win < s.n_fft) ? win : s.n_fft;
    const int pad_w = (s.n_fft - w_len) / 2;
    const int idx = n - pad_w;
    if (idx >= 0 && idx < w_len) {
      const double w = (w_len == 1) ? 1.0 : 0.5 - 0.5 * cospi(2.0 * (double)idx / (double)w_len);
      const long long rr = ((long long)n * bin) % s.n_fft;
      double sn, cs;
      sincospi(2.0 * (double)rr / (double)s.n_fft, &sn, &cs);
      v = part == 0 ? w * cs : -w * sn;
    }
  }
  const __nv_bfloat16 hi = __double2bfloat16(v);
  const __nv_bfloat16 lo = __double2bfloat16(v - (double)__bfloat162float(hi));
  const size_t tile_bytes = (size_t)s.tile_cols * 128;
  char *base = reinterpret_cast<char *>(img) + ((size_t)(nt * s.kchunks + kc) * 2) * tile_bytes;
  *reinterpret_cast<__nv_bfloat16 *>(base + sw128(r, j)) = hi;
  *reinterpret_cast<__nv_bfloat16 *>(base + tile_bytes + sw128(r, j)) = lo;
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier helpers (inline PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major operand, 128-byte swizzle: rows of 128 bytes, 8-row groups 1024
// bytes apart (stride byte offset), sm_100 descriptor version 1.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;            // leading byte offset (unused by swizzled K-major)
  d |= (uint64_t)(1024u >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1u << 46;            // descriptor version
  d |= (uint64_t)2u << 61;            // 128-byte swizzle
  return d;
}

// kind::f16 instruction descriptor: f32 accumulator, bf16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kDftM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase: false after ~2^22 polls (well over a
// second), which the caller turns into an error.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); it++) {
    if (mbar_try_wait(mbar, parity)) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Two bf16 parts of 8 floats, packed for one 16-byte store each.
__device__ __forceinline__ void split8(const float *x, uint4 &hi, uint4 &lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const __nv_bfloat162 a = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
    const float2 af = __bfloat1622float2(a);
    const __nv_bfloat162 b = __floats2bfloat162_rn(x[2 * i] - af.x, x[2 * i + 1] - af.y);
    h[i] = *reinterpret_cast<const uint32_t *>(&a);
    l[i] = *reinterpret_cast<const uint32_t *>(&b);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

constexpr int kDftStages = 2;

// 32 samples (x[first + q], q < 32) of one frame row, with the padding rule
// of sample_at; zeros for frames past the clip.
__device__ __forceinline__ void load_row32(float *x, const float *sig, long long first, long long length,
                                           long long sig_off, int pad_mode, bool valid) {
  if (valid && first >= 0 && first + 32 <= length && ((sig_off + first) & 3) == 0) {
    const float4 *p4 = reinterpret_cast<const float4 *>(sig + first);
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float4 v = __ldg(p4 + q);
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 32; q++) x[q] = valid ? sample_at(sig, first + q, length, pad_mode) : 0.0f;
  }
}

struct DftSmem {
  size_t a_hi[kDftStages], a_lo[kDftStages], b_hi[kDftStages], b_lo[kDftStages];
  size_t w2, seg, bar, taddr, total;
};
__host__ __device__ inline DftSmem dft_smem_layout(const DftShape &s, int n_mels) {
  DftSmem L{};
  size_t p = 0;
  const size_t a_bytes = (size_t)kDftM * 128, b_bytes = ((size_t)s.tile_cols * 128 + 1023) & ~size_t(1023);
  for (int st = 0; st < kDftStages; st++) {
    L.a_hi[st] = p;
    p += a_bytes;
    L.a_lo[st] = p;
    p += a_bytes;
    L.b_hi[st] = p;
    p += b_bytes;
    L.b_lo[st] = p;
    p += b_bytes;
  }
  // the power spectrum of one N tile ([bins][128] floats) reuses the stages
  L.w2 = p;
  p += align16(8 * (size_t)s.nbins);
  L.seg = p;
  p += align16(8 * (size_t)(n_mels + 1));
  L.bar = p;  // full[2], empty[2]
  p += 32;
  L.taddr = p;
  p += 16;
  L.total = p + 1024;  // slack to align the base to 1024 bytes
  return L;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// One arrival that also announces `bytes` of bulk copies completing on the barrier.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared (no multicast), completing on `bar`.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

template <int SPLIT>
__global__ void __launch_bounds__(kDftThreads, 1) dft_gemm_kernel(FrontArgs a, DftShape S, const __nv_bfloat16 *basis,
                                                                   unsigned *err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const DftSmem Ly = dft_smem_layout(S, a.n_mels);
  float *P = reinterpret_cast<float *>(sm);  // [bins of the N tile][128], after its MMAs
  float2 *w2_s = reinterpret_cast<float2 *>(sm + Ly.w2);
  int2 *seg_s = reinterpret_cast<int2 *>(sm + Ly.seg);
  const uint32_t bar0 = smem_u32(sm + Ly.bar);
  auto full_bar = [&](int st) { return bar0 + 8u * (uint32_t)st; };
  auto empty_bar = [&](int st) { return bar0 + 16u + 8u * (uint32_t)st; };
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(sm + Ly.taddr);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int row = tid & (kDftM - 1);  // frame of the tile (= TMEM lane)
  const int half = tid >> 7;          // which 32 columns of a chunk this thread builds
  const int nmel = a.n_mels;
  for (int i = tid; i < S.nbins; i += kDftThreads) w2_s[i] = __ldg(a.mel_w2 + i);
  for (int i = tid; i <= nmel; i += kDftThreads) seg_s[i] = __ldg(a.mel_seg + i);
  if (tid == 0) {
    for (int st = 0; st < kDftStages; st++) {
      mbar_init(full_bar(st), 1);
      mbar_init(empty_bar(st), 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                 "r"(kDftTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;
  const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const uint32_t idesc = idesc_bf16(S.tile_cols);
  const uint32_t b_img = (uint32_t)S.tile_cols * 128u;
  const int seg_lo = seg_s[0].x, seg_hi = seg_s[nmel].x;

  // per-stage state as bits (stage st = bit st): expected phase parities and
  // whether an MMA commit on empty[st] has not been waited for yet
  uint32_t full_ph = 0, empty_ph = 0, pend = 0;
  const size_t stage_stride = Ly.a_hi[1] - Ly.a_hi[0];
  uint32_t chunk = 0;
  bool failed = false, broken = false;
  int cur_clip = -1;
  float vmax = -INFINITY;
  const int total = a.total_tiles;
  const int t_begin = (int)((long long)blockIdx.x * total / gridDim.x);
  const int t_end = (int)((long long)(blockIdx.x + 1) * total / gridDim.x);

  for (int tile = t_begin; tile < t_end && !failed; tile++) {
    const int c = __ldg(a.tile_clip + tile);
    if (c != cur_clip) {
      float m = vmax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if ((tid & 31) == 0 && cur_clip >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur_clip, enc_f(m));
      cur_clip = c;
      vmax = -INFINITY;
    }
    const ClipDesc cd = load_clip(a.clips + c);
    const int t = (tile - cd.tile_base) * kDftM + row;  // this thread's frame
    const bool valid = t < cd.n_frames;
    const float *sig = a.signal + cd.sig_off;
    const long long s0 = (long long)t * a.hop - a.pad + S.k0 + 32 * half;
    float *dst = a.out + (cd.frame_off + t) * (long long)nmel;
    // mel state of this frame (threads of half 0), bins arrive in order across N tiles
    int cur = 0;
    float Rprev = 0.0f, Rcur = 0.0f, Fcur = 0.0f, chk = 0.0f, fmax_ = -INFINITY;
    auto emit = [&](int m, float v) {
      if (seg_s[m].y) v = __int_as_float(0x7fc00000);
      const float val = db10_frame(v, a.amin, 10.0f * log10f(a.ref));
      if (valid) dst[m] = val;
      fmax_ = fmaxf(fmax_, val);
    };
    auto finish_seg = [&]() {
      if (cur >= 1) emit(cur - 1, Rprev + Fcur);
      Rprev = Rcur;
      Rcur = 0.0f;
      Fcur = 0.0f;
      cur++;
    };

    // samples of the next K chunk, loaded one chunk ahead (a chunk's samples
    // are the same for every N tile)
    float xn[32];
    load_row32(xn, sig, s0, cd.length, cd.sig_off, a.pad_mode, valid);
    for (int nt = 0; nt < S.ntiles && !failed; nt++) {
      for (int kc = 0; kc < S.kchunks; kc++) {
        const int st = (int)(chunk & 1u);
        bool ok = true;
        const uint32_t bit = 1u << st;
        if (pend & bit) {  // the MMAs that read this stage two chunks ago are done
          ok = mbar_wait_bounded(empty_bar(st), (empty_ph >> st) & 1u);
          empty_ph ^= bit;
          pend &= ~bit;
        }
        unsigned char *stage = sm + (size_t)st * stage_stride;
        unsigned char *a_hi = stage + Ly.a_hi[0], *a_lo = stage + Ly.a_lo[0];
        unsigned char *b_hi = stage + Ly.b_hi[0], *b_lo = stage + Ly.b_lo[0];
        if (tid == 0 && ok && !broken) {
          const char *src = reinterpret_cast<const char *>(basis) + (size_t)(nt * S.kchunks + kc) * 2 * b_img;
          mbar_expect_tx(full_bar(st), SPLIT == 3 ? 2u * b_img : b_img);
          bulk_g2s(smem_u32(b_hi), src, b_img, full_bar(st));
          if (SPLIT == 3) bulk_g2s(smem_u32(b_lo), src + b_img, b_img, full_bar(st));
        }
        // ---- A chunk: this thread's 32 samples of its frame row
        {
          float x[32];
#pragma unroll
          for (int q = 0; q < 32; q++) x[q] = xn[q];
          const bool last = kc + 1 == S.kchunks && nt + 1 == S.ntiles;
          if (!last) {
            const int kn = kc + 1 < S.kchunks ? kc + 1 : 0;
            load_row32(xn, sig, s0 + (long long)kn * kDftKC, cd.length, cd.sig_off, a.pad_mode, valid);
          }
#pragma unroll
          for (int q = 0; q < 4; q++) {
            uint4 hi, lo;
            split8(x + 8 * q, hi, lo);
            const uint32_t off = sw128(row, 32 * half + 8 * q);
            *reinterpret_cast<uint4 *>(a_hi + off) = hi;
            if (SPLIT == 3) *reinterpret_cast<uint4 *>(a_lo + off) = lo;
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (__syncthreads_or(!ok)) {  // an MMA never completed: every thread decides alike
          failed = true;
          if (tid == 0) atomicOr(err, 1u);
          break;
        }
        if (tid == 0 && !broken) {
          if (mbar_wait_bounded(full_bar(st), (full_ph >> st) & 1u)) {
            tc_fence_after();
            const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
            const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
            for (int kk = 0; kk < kDftKC / 16; kk++) {
              const uint64_t dah = desc_sw128(ah + kk * 32), dbh = desc_sw128(bh + kk * 32);
              umma_bf16(tmem, dah, dbh, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
              if (SPLIT == 3) {
                umma_bf16(tmem, dah, desc_sw128(bl + kk * 32), idesc, 1u);
                umma_bf16(tmem, desc_sw128(al + kk * 32), dbh, idesc, 1u);
              }
            }
            umma_commit(empty_bar(st));
          } else {  // the basis never arrived: no commit, so the others time out on empty[st]
            broken = true;
            atomicOr(err, 1u);
          }
        }
        full_ph ^= bit;
        pend |= bit;
        chunk++;
      }
      if (failed) break;
      // ---- drain: the tile's accumulator is complete
      bool ok = true;
      for (int st = 0; st < kDftStages; st++)
        if (pend & (1u << st)) {
          ok = mbar_wait_bounded(empty_bar(st), (empty_ph >> st) & 1u) && ok;
          empty_ph ^= 1u << st;
          pend &= ~(1u << st);
        }
      if (__syncthreads_or(!ok)) {
        failed = true;
        if (tid == 0) atomicOr(err, 1u);
        break;
      }
      tc_fence_after();
      // ---- |X|^2 of this tile's bins into P[bin][frame]; the two warps of a
      // lane quarter take alternate 16-column pieces
      const int kb = nt * S.tile_cols / 2;
      const int nb = min(S.tile_cols / 2, S.nbins - kb);
      for (int col = 16 * half; col < 2 * nb; col += 32) {
        float v[16];
        tmem_ld16(lane_base + (uint32_t)col, v);
#pragma unroll
        for (int b = 0; b < 8; b++) {
          const int bin = col / 2 + b;
          if (bin < nb) P[bin * kDftM + row] = fmaf(v[2 * b], v[2 * b], v[2 * b + 1] * v[2 * b + 1]);
        }
      }
      __syncthreads();
      if (half == 0) {
        for (int bin = 0; bin < nb; bin++) chk += P[bin * kDftM + row];
        // ---- fold this tile's bins into the mel bands (uniform control flow)
        for (int bin = max(kb, seg_lo); bin < min(kb + nb, seg_hi); bin++) {
          while (cur < nmel && bin >= seg_s[cur + 1].x) finish_seg();
          const float2 w = w2_s[bin];
          const float p = P[(bin - kb) * kDftM + row];
          Rcur = fmaf(w.x, p, Rcur);
          Fcur = fmaf(w.y, p, Fcur);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // P reads before later bulk copies
      tc_fence_before();
      __syncthreads();  // P (aliasing the stages) and the accumulator are free again
    }
    if (failed) break;
    if (half == 0) {
      while (cur < nmel) finish_seg();
      if (nmel > 0) emit(nmel - 1, Rprev);
      if (!isfinite(chk)) {  // a non-finite bin: every band of the frame is NaN -> amin
        const float val = db10_frame(a.amin, a.amin, 10.0f * log10f(a.ref));
        if (valid)
          for (int m = 0; m < nmel; m++) dst[m] = val;
        fmax_ = val;
      }
      if (valid) vmax = fmaxf(vmax, fmax_);
    }
  }
  if (!failed) {
    float m = vmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0 && cur_clip >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur_clip, enc_f(m));
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kDftTmemCols) : "memory");
}

cudaError_t build_dft_basis(__nv_bfloat16 *img, const DftShape &s, int win, int window_zero, cudaStream_t st) {
  const long long total = (long long)s.ntiles * s.kchunks * s.tile_cols * kDftKC;
  build_dft_basis_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(img, s, win, window_zero);
  return cudaGetLastError();
}

cudaError_t launch_dft_gemm(int form, const FrontArgs &a, const DftShape &s, const __nv_bfloat16 *basis,
                            unsigned *err, cudaStream_t st, int *launched) {
  if (launched) *launched = 0;
  if (a.total_tiles <= 0) return cudaSuccess;
  if (!a.mel_seg_ok) return cudaErrorInvalidValue;  // the epilogue needs the per-bin split
  const size_t smem = std::max(dft_smem_layout(s, a.n_mels).total, kDftMinSmem);
  const void *kern = form == DFT_GEMM_BF16X3 ? reinterpret_cast<const void *>(dft_gemm_kernel<3>)
                                              : reinterpret_cast<const void *>(dft_gemm_kernel<1>);
  int per_sm = 1, sms = 148;
  cudaError_t e = persistent_geometry(kern, kDftThreads, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  per_sm = std::min(per_sm, 512 / kDftTmemCols);
  long long grid = (long long)sms * per_sm;
  if (grid > a.total_tiles) grid = a.total_tiles;
  if (form == DFT_GEMM_BF16X3)
    dft_gemm_kernel<3><<<(unsigned)grid, kDftThreads, smem, st>>>(a, s, basis, err);
  else
    dft_gemm_kernel<1><<<(unsigned)grid, kDftThreads, smem, st>>>(a, s, basis, err);
  if (launched) *launched = (int)grid;
  return cudaGetLastError();
}

}  // namespace mm
