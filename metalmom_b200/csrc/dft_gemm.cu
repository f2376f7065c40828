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
// One CTA per SM (it holds all 512 TMEM columns), warp-specialised, with
// mbarriers between the roles instead of block-wide barriers:
//  * 16 producer warps: four threads per frame row convert 16 samples each of
//    the K chunk (64 samples) into bf16 hi/lo in the K-major 128-byte-swizzle
//    layout of the A ring (2 stages), with the samples of the next two chunks
//    already loading; producer thread 0 also moves each basis chunk (a
//    pre-swizzled image, hi and lo) into the B ring (3 stages where shared
//    memory allows, 2 otherwise) by bulk async copies;
//  * one MMA thread: per chunk 4 (bf16) or 12 (bf16x3) tcgen05.mma of
//    M 128 x N tile_cols x K 16 into one of two TMEM accumulators, committed
//    to the stages' "empty" barriers and, after the last chunk of an N tile,
//    to the accumulator's "full" barrier;
//  * 4 epilogue warps (TMEM lane quarters): while the next N tile fills the
//    other accumulator, each thread reads its frame's columns (tcgen05.ld),
//    forms |X|^2 and folds the bins into the mel bands with the per-bin split
//    of the filterbank (band m = R[m] + F[m+1]); the log-mel row and the clip
//    maximum are written as by the FFT kernels, and the same DCT kernel
//    follows.
//
// Every wait is bounded: a wait that runs out sets the error word and the
// CTA stops, releases its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "async_copy.cuh"
#include "tcgen05.cuh"
#include "frame_common.cuh"
#include "kernels.h"

namespace mm {

constexpr int kDftM = 128;   // frames per tile = TMEM lanes
constexpr int kDftKC = 64;   // K per chunk: one 128-byte swizzle row of bf16
// Warp roles: 16 producer warps (four threads per frame row build the A
// chunk, 16 samples each, two chunks of samples in flight), 4 epilogue warps
// (warp 16 + q reads TMEM lane quarter q), 1 MMA warp.
constexpr int kDftRowSplit = 4;
constexpr int kDftRowCols = kDftKC / kDftRowSplit;  // 16 samples per producer thread
constexpr int kDftProducers = kDftM * kDftRowSplit;
constexpr int kDftEpiWarp0 = kDftProducers / 32;
constexpr int kDftMmaWarp = kDftEpiWarp0 + 4;
constexpr int kDftThreads = 32 * (kDftMmaWarp + 1);
constexpr int kDftTmemCols = 512;  // two accumulators of up to 256 columns
constexpr int kDftAStages = 2;     // A chunks: built on the SM, quickly

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

// Two 16-bit parts of a float64 value: v ~ hi + lo (bf16 or fp16).
__device__ __forceinline__ void split_parts(double v, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
  hi = __double2bfloat16(v);
  lo = __double2bfloat16(v - (double)__bfloat162float(hi));
}
__device__ __forceinline__ void split_parts(double v, __half &hi, __half &lo) {
  hi = __double2half(v);
  lo = __double2half(v - (double)__half2float(hi));
}

// B image: [tile][chunk][part hi/lo][tile_cols rows x 128 bytes], values in
// float64 (window and twiddle), split into two 16-bit parts (T: bf16 or fp16;
// the fp16 parts of values up to 1 lose nothing to range: lo parts below
// fp16's normal range keep an absolute precision of 2^-24).
template <typename T>
__global__ void build_dft_basis_kernel(T *img, DftShape s, int win, int window_zero) {
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
  T hi, lo;
  split_parts(v, hi, lo);
  const size_t tile_bytes = (size_t)s.tile_cols * 128;
  char *base = reinterpret_cast<char *>(img) + ((size_t)(nt * s.kchunks + kc) * 2) * tile_bytes;
  *reinterpret_cast<T *>(base + sw128(r, j)) = hi;
  *reinterpret_cast<T *>(base + tile_bytes + sw128(r, j)) = lo;
}

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier helpers (inline PTX)
// ---------------------------------------------------------------------------
// Two 16-bit parts (bf16, or fp16 when F16) of 8 floats, packed for one
// 16-byte store each.
template <bool F16>
__device__ __forceinline__ void split8(const float *x, uint4 &hi, uint4 &lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    if constexpr (F16) {
      const __half2 a = __floats2half2_rn(x[2 * i], x[2 * i + 1]);
      const float2 af = __half22float2(a);
      const __half2 b = __floats2half2_rn(x[2 * i] - af.x, x[2 * i + 1] - af.y);
      h[i] = *reinterpret_cast<const uint32_t *>(&a);
      l[i] = *reinterpret_cast<const uint32_t *>(&b);
    } else {
      const __nv_bfloat162 a = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
      const float2 af = __bfloat1622float2(a);
      const __nv_bfloat162 b = __floats2bfloat162_rn(x[2 * i] - af.x, x[2 * i + 1] - af.y);
      h[i] = *reinterpret_cast<const uint32_t *>(&a);
      l[i] = *reinterpret_cast<const uint32_t *>(&b);
    }
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}


// NS samples (x[first + q], q < NS) of one frame row, with the padding rule
// of sample_at; zeros for frames past the clip.
template <int NS>
__device__ __forceinline__ void load_row(float *x, const float *sig, long long first, long long length,
                                         long long sig_off, int pad_mode, bool valid) {
  if (valid && first >= 0 && first + NS <= length && ((sig_off + first) & 3) == 0) {
    const float4 *p4 = reinterpret_cast<const float4 *>(sig + first);
#pragma unroll
    for (int q = 0; q < NS / 4; q++) {
      const float4 v = __ldg(p4 + q);
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < NS; q++) x[q] = valid ? sample_at(sig, first + q, length, pad_mode) : 0.0f;
  }
}

// Shared memory: the A ring (hi, lo), the B ring (hi, lo: basis chunks by
// bulk copy; three stages when they fit, to cover the L2 latency), the
// per-bin filterbank split and the barriers.
struct DftSmem {
  int b_stages;
  size_t a0, a_stage, b0, b_stage, b_img, w2, seg, bar, taddr, total;
};
__host__ __device__ inline DftSmem dft_smem_layout(const DftShape &s, int n_mels) {
  DftSmem L{};
  const size_t a_img = (size_t)kDftM * 128;
  L.b_img = ((size_t)s.tile_cols * 128 + 1023) & ~size_t(1023);
  L.a_stage = 2 * a_img;
  L.b_stage = 2 * L.b_img;
  const size_t tail = align16(8 * (size_t)s.nbins) + align16(8 * (size_t)(n_mels + 1)) + 256 + 1024;
  L.b_stages = (kDftAStages * L.a_stage + 3 * L.b_stage + tail <= 227 * 1024) ? 3 : 2;
  size_t p = 0;
  L.a0 = p;
  p += kDftAStages * L.a_stage;
  L.b0 = p;
  p += (size_t)L.b_stages * L.b_stage;
  L.w2 = p;
  p += align16(8 * (size_t)s.nbins);
  L.seg = p;
  p += align16(8 * (size_t)(n_mels + 1));
  L.bar = p;  // a_full[2] a_empty[2] b_full[3] b_empty[3] acc_full[2] acc_empty[2] fin
  p += 8 * 16;
  L.taddr = p;
  p += 16;
  L.total = p + 1024;  // slack to align the base to 1024 bytes
  return L;
}

// F16: fp16 parts, with each frame's samples scaled by a.frame_scale (a power
// of two, so that the frame's largest sample is in [0.5, 1)) before the
// split and |X|^2 scaled back exactly in the epilogue.
template <int SPLIT, bool F16>
__global__ void __launch_bounds__(kDftThreads, 1) dft_gemm_kernel(FrontArgs a, DftShape S, const void *basis,
                                                                   unsigned *err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  unsigned char *sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
  const DftSmem Ly = dft_smem_layout(S, a.n_mels);
  const int SB = Ly.b_stages;
  float2 *w2_s = reinterpret_cast<float2 *>(sm + Ly.w2);
  int2 *seg_s = reinterpret_cast<int2 *>(sm + Ly.seg);
  const uint32_t bar0 = smem_u32(sm + Ly.bar);
  auto a_full = [&](int st) { return bar0 + 8u * (uint32_t)st; };
  auto a_empty = [&](int st) { return bar0 + 16u + 8u * (uint32_t)st; };
  auto b_full = [&](int st) { return bar0 + 32u + 8u * (uint32_t)st; };
  auto b_empty = [&](int st) { return bar0 + 56u + 8u * (uint32_t)st; };
  auto acc_full = [&](int b) { return bar0 + 80u + 8u * (uint32_t)b; };
  auto acc_empty = [&](int b) { return bar0 + 96u + 8u * (uint32_t)b; };
  const uint32_t fin = bar0 + 112u;
  uint32_t *taddr_s = reinterpret_cast<uint32_t *>(sm + Ly.taddr);
  const uint32_t b_img = (uint32_t)S.tile_cols * 128u;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nmel = a.n_mels;
  for (int i = tid; i < S.nbins; i += kDftThreads) w2_s[i] = __ldg(a.mel_w2 + i);
  for (int i = tid; i <= nmel; i += kDftThreads) seg_s[i] = __ldg(a.mel_seg + i);
  if (tid == 0) {
    for (int st = 0; st < kDftAStages; st++) {
      mbar_init(a_full(st), kDftProducers);
      mbar_init(a_empty(st), 1);
    }
    for (int st = 0; st < SB; st++) {
      mbar_init(b_full(st), 1);
      mbar_init(b_empty(st), 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(acc_full(b), 1);
      mbar_init(acc_empty(b), kDftM);
    }
    mbar_init(fin, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kDftMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                 "r"(kDftTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;
  const int total = a.total_tiles;
  const int t_begin = (int)((long long)blockIdx.x * total / gridDim.x);
  const int t_end = (int)((long long)(blockIdx.x + 1) * total / gridDim.x);

  if (warp < kDftEpiWarp0) {
    // ---------------- producers: A chunks (and thread 0: the basis chunks)
    const int row = tid & (kDftM - 1), part = tid >> 7;  // 16 columns of the chunk per thread
    uint32_t c = 0;  // chunk counter (A ring stage c % 2, B ring stage c % SB)
    bool ok = true;
    for (int tile = t_begin; tile < t_end && ok; tile++) {
      const int cl = __ldg(a.tile_clip + tile);
      const ClipDesc cd = load_clip(a.clips + cl);
      const int t = (tile - cd.tile_base) * kDftM + row;
      const bool valid = t < cd.n_frames;
      const float *sig = a.signal + cd.sig_off;
      const long long s0 = (long long)t * a.hop - a.pad + S.k0 + kDftRowCols * part;
      const float sc = (F16 && valid) ? __ldg(a.frame_scale + cd.frame_off + t) : 1.0f;
      // samples two chunks ahead (a chunk's samples serve every N tile)
      const int nchunks = S.ntiles * S.kchunks;
      float xn[kDftRowCols], xn2[kDftRowCols];
      load_row<kDftRowCols>(xn, sig, s0, cd.length, cd.sig_off, a.pad_mode, valid);
      load_row<kDftRowCols>(xn2, sig, s0 + (long long)(1 % S.kchunks) * kDftKC, cd.length, cd.sig_off,
                            a.pad_mode, valid && nchunks > 1);
      for (int nt = 0; nt < S.ntiles && ok; nt++) {
        for (int kc = 0; kc < S.kchunks && ok; kc++, c++) {
          const int sa = (int)(c % kDftAStages), sb = (int)(c % (uint32_t)SB);
          const uint32_t pa = (c / kDftAStages) & 1u, pb = (c / (uint32_t)SB) & 1u;
          if (tid == 0) {  // the basis chunk of (nt, kc) into B stage sb
            if (!mbar_wait_bounded(b_empty(sb), pb ^ 1u)) {
              ok = false;
              atomicOr(err, 1u);
              break;
            }
            unsigned char *bs = sm + Ly.b0 + (size_t)sb * Ly.b_stage;
            const char *src = static_cast<const char *>(basis) + (size_t)(nt * S.kchunks + kc) * 2 * b_img;
            mbar_expect_tx(b_full(sb), SPLIT == 3 ? 2u * b_img : b_img);
            bulk_g2s(smem_u32(bs), src, b_img, b_full(sb));
            if (SPLIT == 3) bulk_g2s(smem_u32(bs + Ly.b_img), src + b_img, b_img, b_full(sb));
          }
          float x[kDftRowCols];
#pragma unroll
          for (int q = 0; q < kDftRowCols; q++) {
            x[q] = xn[q];
            xn[q] = xn2[q];
          }
          const int ci = nt * S.kchunks + kc;
          if (ci + 2 < nchunks)
            load_row<kDftRowCols>(xn2, sig, s0 + (long long)((kc + 2) % S.kchunks) * kDftKC, cd.length, cd.sig_off,
                                  a.pad_mode, valid);
          if (!mbar_wait_bounded(a_empty(sa), pa ^ 1u)) {
            ok = false;
            atomicOr(err, 1u);
            break;
          }
          unsigned char *as = sm + Ly.a0 + (size_t)sa * Ly.a_stage;
#pragma unroll
          for (int q = 0; q < kDftRowCols / 8; q++) {
            uint4 hi, lo;
            if constexpr (F16) {
              float xs[8];
#pragma unroll
              for (int u = 0; u < 8; u++) xs[u] = x[8 * q + u] * sc;
              split8<true>(xs, hi, lo);
            } else {
              split8<false>(x + 8 * q, hi, lo);
            }
            const uint32_t off = sw128(row, kDftRowCols * part + 8 * q);
            *reinterpret_cast<uint4 *>(as + off) = hi;
            if (SPLIT == 3) *reinterpret_cast<uint4 *>(as + kDftM * 128 + off) = lo;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(a_full(sa));
        }
      }
    }
    // bulk copies still in flight write into this CTA's shared memory: wait
    // for the ones armed last (their phases complete once the bytes land)
    if (tid == 0)
      for (uint32_t q = c > (uint32_t)SB ? c - SB : 0; q < c; q++)
        mbar_wait_bounded(b_full((int)(q % (uint32_t)SB)), (q / (uint32_t)SB) & 1u);
  } else if (warp == kDftMmaWarp) {
    // ---------------- MMA issue (one thread)
    if (lane == 0) {
      const uint32_t idesc = idesc_f16kind<F16>(S.tile_cols, kDftM);
      uint32_t c = 0, j = 0;  // chunk and accumulator-tile counters
      bool ok = true;
      for (int tile = t_begin; tile < t_end && ok; tile++) {
        for (int nt = 0; nt < S.ntiles && ok; nt++, j++) {
          const int ab = (int)(j & 1u);
          if (!mbar_wait_bounded(acc_empty(ab), ((j >> 1) & 1u) ^ 1u)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t acc = tmem + (uint32_t)ab * 256u;
          for (int kc = 0; kc < S.kchunks; kc++, c++) {
            const int sa = (int)(c % kDftAStages), sb = (int)(c % (uint32_t)SB);
            if (!mbar_wait_bounded(a_full(sa), (c / kDftAStages) & 1u) ||
                !mbar_wait_bounded(b_full(sb), (c / (uint32_t)SB) & 1u)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t ah = smem_u32(sm + Ly.a0 + (size_t)sa * Ly.a_stage), al = ah + kDftM * 128;
            const uint32_t bh = smem_u32(sm + Ly.b0 + (size_t)sb * Ly.b_stage), bl = bh + (uint32_t)Ly.b_img;
#pragma unroll
            for (int kk = 0; kk < kDftKC / 16; kk++) {
              const uint64_t dah = desc_sw128(ah + kk * 32), dbh = desc_sw128(bh + kk * 32);
              umma_f16kind(acc, dah, dbh, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
              if (SPLIT == 3) {
                umma_f16kind(acc, dah, desc_sw128(bl + kk * 32), idesc, 1u);
                umma_f16kind(acc, desc_sw128(al + kk * 32), dbh, idesc, 1u);
              }
            }
            umma_commit(a_empty(sa));  // the stages are free once these MMAs complete
            umma_commit(b_empty(sb));
          }
          if (ok) umma_commit(acc_full(ab));
        }
      }
      if (!ok) atomicOr(err, 1u);
      umma_commit(fin);  // every MMA issued here has completed once this arrives
      mbar_wait_bounded(fin, 0u);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue: |X|^2 of each N tile and the mel fold, one frame per thread
    const int row = 32 * (warp & 3) + lane;  // TMEM lane = frame of the tile
    const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const int seg_lo = seg_s[0].x, seg_hi = seg_s[nmel].x;
    const float ref_db = 10.0f * log10f(a.ref);
    uint32_t j = 0;
    bool ok = true;
    int cur_clip = -1;
    float vmax = -INFINITY;
    for (int tile = t_begin; tile < t_end && ok; tile++) {
      const int cl = __ldg(a.tile_clip + tile);
      if (cl != cur_clip) {
        float m = vmax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0 && cur_clip >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur_clip, enc_f(m));
        cur_clip = cl;
        vmax = -INFINITY;
      }
      const ClipDesc cd = load_clip(a.clips + cl);
      const int t = (tile - cd.tile_base) * kDftM + row;
      const bool valid = t < cd.n_frames;
      float *dst = a.out + (cd.frame_off + t) * (long long)nmel;
      float isc2 = 1.0f;  // F16: 1 / scale^2, a power of two (exact)
      if constexpr (F16) {
        const float sc = valid ? __ldg(a.frame_scale + cd.frame_off + t) : 1.0f;
        isc2 = 1.0f / (sc * sc);
      }
      int cur = 0;
      float Rprev = 0.0f, Rcur = 0.0f, Fcur = 0.0f, chk = 0.0f, fmax_ = -INFINITY;
      auto emit = [&](int m, float v) {
        if constexpr (F16) v *= isc2;
        if (seg_s[m].y) v = __int_as_float(0x7fc00000);
        const float val = db10_frame(v, a.amin, ref_db);
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
      for (int nt = 0; nt < S.ntiles; nt++, j++) {
        const int ab = (int)(j & 1u);
        if (!mbar_wait_bounded(acc_full(ab), (j >> 1) & 1u)) {
          ok = false;
          atomicOr(err, 1u);
          break;
        }
        tc_fence_after();
        const int kb = nt * S.tile_cols / 2;
        const int nb = min(S.tile_cols / 2, S.nbins - kb);
        for (int col = 0; col < 2 * nb; col += 16) {
          float v[16];
          tmem_ld16(lane_base + (uint32_t)ab * 256u + (uint32_t)col, v);
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const int bin = kb + col / 2 + q;
            if (bin >= kb + nb) break;
            const float p = fmaf(v[2 * q], v[2 * q], v[2 * q + 1] * v[2 * q + 1]);
            chk = fmaf(p, 0.0f, chk);  // NaN iff a bin is not finite
            if (bin < seg_lo || bin >= seg_hi) continue;
            while (cur < nmel && bin >= seg_s[cur + 1].x) finish_seg();
            const float2 w = w2_s[bin];
            Rcur = fmaf(w.x, p, Rcur);
            Fcur = fmaf(w.y, p, Fcur);
          }
        }
        tc_fence_before();
        mbar_arrive(acc_empty(ab));  // the accumulator may take the next N tile after next
      }
      if (!ok) break;
      while (cur < nmel) finish_seg();
      if (nmel > 0) emit(nmel - 1, Rprev);
      if (!isfinite(chk)) {  // a non-finite bin: every band of the frame is NaN -> amin
        const float val = db10_frame(a.amin, a.amin, ref_db);
        if (valid)
          for (int m = 0; m < nmel; m++) dst[m] = val;
        fmax_ = val;
      }
      if (valid) vmax = fmaxf(vmax, fmax_);
    }
    if (ok) {
      float m = vmax;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0 && cur_clip >= 0 && m > -INFINITY) atomicMax(a.clip_max + cur_clip, enc_f(m));
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kDftMmaWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kDftTmemCols) : "memory");
}

cudaError_t build_dft_basis(void *img, const DftShape &s, int win, int window_zero, bool f16, cudaStream_t st) {
  const long long total = (long long)s.ntiles * s.kchunks * s.tile_cols * kDftKC;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  if (f16)
    build_dft_basis_kernel<__half><<<blocks, 256, 0, st>>>(static_cast<__half *>(img), s, win, window_zero);
  else
    build_dft_basis_kernel<__nv_bfloat16><<<blocks, 256, 0, st>>>(static_cast<__nv_bfloat16 *>(img), s, win,
                                                                   window_zero);
  return cudaGetLastError();
}

// Per frame: 2^-e with 2^(e-1) <= max |x| < 2^e over the samples the frame's
// DFT reads (the window's support, s.k0 .. s.k0 + s.kw), so the scaled
// samples lie in (-1, 1) and their fp16 lo parts keep 2^-24 of the frame's
// largest sample even where they fall below fp16's normal range.  Frames that
// reach into the padding take the maximum over a range that covers every
// sample the padding rule (zeros or a mirror) can read.  A frame of zeros, or
// one holding a non-finite sample, gets 1 (the non-finite value then reaches
// the spectrum, as in the FFT form).  e is clamped to [-63, 63] so that the
// epilogue's 1 / scale^2 is a normal float.  One warp per frame.
__global__ void frame_scale_kernel(FrontArgs a, DftShape s, float *scale) {
  const int lane = threadIdx.x & 31;
  const int warps = (blockDim.x >> 5) * gridDim.x;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (long long w = w0; w < (long long)a.total_tiles * kDftM; w += warps) {
    const int tile = (int)(w / kDftM), row = (int)(w - (long long)tile * kDftM);
    const int cl = __ldg(a.tile_clip + tile);
    const ClipDesc cd = load_clip(a.clips + cl);
    const int t = (tile - cd.tile_base) * kDftM + row;
    if (t >= cd.n_frames) continue;  // warp-uniform
    const float *sig = a.signal + cd.sig_off;
    long long lo = (long long)t * a.hop - a.pad + s.k0, hi = lo + s.kw;
    if (lo < 0 || hi > cd.length) {  // mirrored samples lie within kw of the edge they mirror
      lo = lo - s.kw;
      hi = hi + s.kw;
    }
    lo = lo < 0 ? 0 : lo;
    hi = hi > cd.length ? cd.length : hi;
    float m = 0.0f;
    bool bad = false;
    for (long long i = lo + lane; i < hi; i += 32) {
      const float v = __ldg(sig + i);
      bad |= !isfinite(v);
      m = fmaxf(m, fabsf(v));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    bad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      float sc = 1.0f;
      if (!bad && m > 0.0f) {
        int e = ilogbf(m) + 1;  // 2^(e-1) <= m < 2^e
        e = e < -63 ? -63 : (e > 63 ? 63 : e);
        sc = ldexpf(1.0f, -e);
      }
      scale[cd.frame_off + t] = sc;
    }
  }
}

cudaError_t launch_frame_scale(const FrontArgs &a, const DftShape &s, cudaStream_t st) {
  if (a.total_tiles <= 0 || !a.frame_scale) return cudaSuccess;
  const long long warps = (long long)a.total_tiles * kDftM;
  const long long blocks = std::min<long long>((warps + 7) / 8, 148LL * 16);
  frame_scale_kernel<<<(unsigned)blocks, 256, 0, st>>>(a, s, const_cast<float *>(a.frame_scale));
  return cudaGetLastError();
}

cudaError_t launch_dft_gemm(int form, const FrontArgs &a, const DftShape &s, const void *basis,
                            unsigned *err, cudaStream_t st, int *launched) {
  if (launched) *launched = 0;
  if (a.total_tiles <= 0) return cudaSuccess;
  if (!a.mel_seg_ok) return cudaErrorInvalidValue;  // the epilogue needs the per-bin split
  if (s.tile_cols > 256) return cudaErrorInvalidValue;
  if (form == DFT_GEMM_F16X3 && !a.frame_scale) return cudaErrorInvalidValue;
  const size_t smem = dft_smem_layout(s, a.n_mels).total;
  const void *kern = form == DFT_GEMM_BF16X3   ? reinterpret_cast<const void *>(dft_gemm_kernel<3, false>)
                     : form == DFT_GEMM_F16X3 ? reinterpret_cast<const void *>(dft_gemm_kernel<3, true>)
                                              : reinterpret_cast<const void *>(dft_gemm_kernel<1, false>);
  int per_sm = 1, sms = 148;
  cudaError_t e = persistent_geometry(kern, kDftThreads, smem, &per_sm, &sms);
  if (e != cudaSuccess) return e;
  long long grid = sms;  // one CTA per SM: it holds all 512 TMEM columns
  if (grid > a.total_tiles) grid = a.total_tiles;
  if (form == DFT_GEMM_BF16X3)
    dft_gemm_kernel<3, false><<<(unsigned)grid, kDftThreads, smem, st>>>(a, s, basis, err);
  else if (form == DFT_GEMM_F16X3)
    dft_gemm_kernel<3, true><<<(unsigned)grid, kDftThreads, smem, st>>>(a, s, basis, err);
  else
    dft_gemm_kernel<1, false><<<(unsigned)grid, kDftThreads, smem, st>>>(a, s, basis, err);
  if (launched) *launched = (int)grid;
  return cudaGetLastError();
}

}  // namespace mm
