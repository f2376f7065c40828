// Interfaces between the host runtime (mm_runtime.cpp / mm_abi.cpp) and the
// CUDA kernels (frontend_kernels.cu).  Plain structs and pointers only.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mm {

// One clip of a batch, as the frame kernels see it.
struct ClipDesc {
  long long sig_off;    // first sample of the clip in the signal buffer
  long long length;     // samples in the clip
  long long frame_off;  // global index of the clip's first frame (frame-major buffers)
  long long out_off;    // element offset of the clip's [rows x n_frames] output block
  int n_frames;         // frames of this clip (reference frame count)
  int tile_base;        // first frame-tile index of this clip
};

enum FrontMode : int {
  MODE_SPECTRUM = 0,  // |X|^power per bin -> out[k][t]          (mm_stft)
  MODE_MEL = 1,       // mel of |X|^power  -> out[m][t]           (mm_mel_spectrogram)
  MODE_MELDB = 2,     // 10 log10(max(mel,amin)/ref) -> out[frame][m] + per-clip max
  MODE_COMPLEX = 3,   // X[k] as (re, im)  -> out[k][t][2]        (mm_stft_complex)
};

// Modes that project onto the mel filterbank (the others write bins).
__host__ __device__ constexpr bool mode_has_mel(int mode) { return mode == MODE_MEL || mode == MODE_MELDB; }

enum PadMode : int { PAD_CONSTANT = 0, PAD_REFLECT = 1 };

// How the spectrum is computed (MMFrontEndParams.dft_form).
enum DftForm : int { DFT_FFT_F32 = 0, DFT_GEMM_BF16X3 = 1, DFT_GEMM_BF16 = 2, DFT_GEMM_F16X3 = 3 };

// Geometry of the DFT-as-GEMM form: bins, N tiles of tile_cols columns
// (cos / -sin per bin), the window support [k0, k0 + kw) cut into K chunks.
struct DftShape {
  int n_fft, nbins, ntiles, tile_cols, k0, kw, kchunks;
};

// Device tables for one (sr, n_fft, win, n_mels, fmin, fmax, n_mfcc) group.
struct DevTables {
  int n_fft = 0, n_mels = 0, n_mfcc = 0;
  float *window = nullptr;   // [n_fft] analysis window (float64-built)
  float2 *tw_stage = nullptr;  // per-stage Stockham twiddles (layout: stage_twiddle_count)
  float2 *tw_split = nullptr;  // exp(-2 pi i k / n_fft), k < n_fft/4 (real split)
  float2 *tw_tiny = nullptr;   // exp(-2 pi i t / n_fft), t < n_fft (n_fft <= 16 only)
  float *mel_w = nullptr;      // dense [n_mels][n_fft/2+1] float32 weights (build stage)
  float *mel_pw = nullptr;     // packed nonzero weights, row after row
  int4 *mel_info = nullptr;    // per mel {start bin, count, packed offset, nan-row flag}
  int mel_nnz = 0;             // entries of mel_pw
  // Per-bin split of the same filterbank (warp kernel): bin k feeds band s(k)
  // with mel_w2[k].x and band s(k)-1 with mel_w2[k].y.  Segment s = the bins
  // [mel_seg[s].x, mel_seg[s+1].x) (n_mels + 1 entries; .y = NaN-row flag of
  // band s).
  float2 *mel_w2 = nullptr;
  int2 *mel_seg = nullptr;
  int mel_seg_ok = 0;          // 0: the split does not describe the filterbank (use mel_pw)
  // Lane tables of the same split for the warp kernel (n_fft 256..2048): lane
  // l of a frame owns bins [32 l, 32 l + 32) and sums them into per-segment
  // parts (layout at build_mel_lane_kernel).
  float2 *mel_lw = nullptr;    // [33][n_fft/64] weights, lane-minor
  int2 *mel_lane = nullptr;    // per lane {flush mask, first slot | chain length | zero slot}
  int *mel_band = nullptr;     // per band: head slot of m | head slot of m+1 | NaN flag
  int mel_lane_ok = 0;
  // DFT-as-GEMM form only: the windowed DFT basis as hi/lo images (bf16, or
  // fp16 for DFT_GEMM_F16X3) and an error word the kernel sets when a bounded
  // wait runs out.
  void *dft_basis = nullptr;
  DftShape dft{};
  unsigned *dft_err = nullptr;
  float *dct = nullptr;        // [n_mfcc_eff][n_mels] DCT-II ortho basis
};

struct FrontArgs {
  const float *signal;
  const ClipDesc *clips;
  const int *tile_clip;  // frame tile -> clip index
  int total_tiles;
  int hop, pad, pad_mode;
  const float *window;
  const float2 *tw_stage;
  const float2 *tw_split;
  const float2 *tw_tiny;
  const int4 *mel_info;
  const float *mel_pw;  // packed weights (mel_info[m].z = offset of row m)
  int mel_nnz;
  const float2 *mel_w2;  // per-bin split (see DevTables)
  const int2 *mel_seg;
  int mel_seg_ok;
  const float2 *mel_lw;  // lane tables (see DevTables)
  const int2 *mel_lane;
  const int *mel_band;
  int mel_lane_ok;
  int n_mels;
  float power;  // exponent applied to |X| (2 = power spectrum)
  float amin, ref;
  float *out;
  unsigned *clip_max;  // MODE_MELDB: order-preserving encoded max per clip
  // DFT_GEMM_F16X3 only: per frame (frame-major, as the log-mel rows) the
  // power of two the frame's samples are scaled by before the fp16 split
  float *frame_scale = nullptr;
  // error word of kernels with bounded waits (tensor-core frame kernel)
  unsigned *err = nullptr;
};

struct DctArgs {
  const float *mel_db;  // [total_frames][n_mels]
  const ClipDesc *clips;
  const int *tile_clip;  // DCT tile (kDctTile frames) -> clip
  const int *tile_first; // first frame (within the clip) of each DCT tile
  int total_tiles;
  const unsigned *clip_max;
  const float *basis;  // [n_mfcc][n_mels]
  int n_mels, n_mfcc;
  float top_db;  // <= 0: no floor
  float *out;    // per clip [n_mfcc][n_frames] at clips[c].out_off
};

constexpr int kDctTile = 64;  // frames per DCT tile (also the onset kernel's tile)

// What follows the log-mel rows on the MFCC path.
enum PostStage : int { POST_DCT = 0, POST_ONSET_MEAN = 1, POST_ONSET_BANDS = 2 };

// Onset strength from the frame-major log-mel: out[o] (or out[b][o]) for
// o = i + shift is the mean over bands (or per band) of
// max(0, S[i+lag][b] - S[i][b]), S floored at max - top_db; 0 elsewhere.
struct OnsetArgs {
  const float *mel_db;
  const ClipDesc *clips;
  const int *tile_clip, *tile_first;
  int total_tiles;
  const unsigned *clip_max;
  int n_mels, lag, shift, bands;
  float top_db;
  float *out;
};
cudaError_t launch_onset(const OnsetArgs &a, cudaStream_t s);

// Savitzky-Golay delta along time of a [n_features x n_frames] matrix
// (interp edges) and stacked delayed copies (zeros before the start).
constexpr int kDeltaMaxWidth = 63;
struct DeltaCoeffs {
  float c[kDeltaMaxWidth];
};
cudaError_t launch_delta(const float *x, float *y, int n_features, int n_frames, int width, DeltaCoeffs c,
                         cudaStream_t s);
cudaError_t launch_stack_memory(const float *x, float *y, int n_features, int n_frames, int n_steps, int delay,
                                cudaStream_t s);

// Frames per CTA tile for a given log2(n_fft) and launch variant.
int frames_per_tile(int log2n, int variant);
// Number of launch variants the autotuner may choose from (1 = not tunable).
int frame_variants(int log2n, int mode, int power_is_2);
// Launch variant 3: the warp-per-frame kernel (MODE_MELDB, n_fft 256..2048).
constexpr int kWarpVariant = 3;
// Launch variant of the tensor-core frame kernel (n_fft 2048, MFCC path):
// both 32-point DFT stages as fp16x3 tcgen05 GEMMs, 16 frames per tile.
constexpr int kTcVariant = 5;
constexpr int kTcFramesPerTile = 16;
int warp_frames_per_tile(int log2n);  // 0 when the size has no warp kernel
// Walking lanes of the filterbank walk (n_fft / 64, 32 bins each) for n_fft
// 256..4096, else 0: the warp kernel's lanes (up to 2048), or the first
// n_fft / 64 threads of a frame in the CTA-tile kernel.
inline int mel_lane_tpf(int n_fft) {
  return (n_fft >= 256 && n_fft <= 4096 && (n_fft & (n_fft - 1)) == 0) ? n_fft / 64 : 0;
}
// Filterbank part slots that fit behind the padded spectrum (ps tpf floats,
// ps = 36 for tpf = 32 and 33 below): in a warp-kernel frame buffer (at
// least 66 tpf floats, frame group g starting tpf g floats in) for tpf <= 32
// (480 at tpf 32, also within the CTA-tile and tensor-core kernels' larger
// buffers); 1024
// (the slot field's range) for tpf = 64, whose CTA-tile frame buffer holds
// more than 33 tpf + 2048 floats.
inline int mel_lane_max_slots(int tpf) {
  if (tpf <= 0) return 0;
  if (tpf > 32) return 1024;
  const int ps = tpf == 32 ? 36 : 33;
  return (66 * tpf - ps * tpf - tpf * (32 / tpf - 1)) / 2;
}
cudaError_t launch_frontend_tc(const FrontArgs &a, int grid_limit, cudaStream_t s, int *launched);
cudaError_t launch_frontend_warp(int log2n, const FrontArgs &a, int grid_limit, cudaStream_t s,
                                 int *launched);
// Stockham twiddle table length (entries) for log2(n_fft) >= 5.
int stage_twiddle_count(int log2n);

// Table construction (float64 math on the device, stored as float32).
cudaError_t build_tables(DevTables &t, int sr, int n_fft, int win, int n_mels, float fmin,
                         float fmax, int n_mfcc_eff, int window_zero, cudaStream_t s);

// The same tables placed in caller-provided device memory [base, base+cap)
// (no allocation); cudaErrorMemoryAllocation when they do not fit, *used =
// bytes taken (256-byte aligned).
cudaError_t build_tables_at(DevTables &t, char *base, size_t cap, size_t *used, int sr, int n_fft,
                            int win, int n_mels, float fmin, float fmax, int n_mfcc_eff, int window_zero,
                            cudaStream_t s);

// Blocks per SM and SM count for a persistent launch of `kern` (cached).
cudaError_t persistent_geometry(const void *kern, int threads, size_t smem, int *per_sm, int *sms);

// DFT-as-GEMM (tcgen05) form: n_fft 256..1024, window no longer than n_fft.
constexpr int kDftVariant = 4;  // launch "variant" of such groups (128-frame tiles)
bool dft_supported(int n_fft, int win);
DftShape dft_shape(int n_fft, int win);
size_t dft_basis_bytes(const DftShape &s);
cudaError_t build_dft_basis(void *img, const DftShape &s, int win, int window_zero, bool f16, cudaStream_t st);
cudaError_t launch_dft_gemm(int form, const FrontArgs &a, const DftShape &s, const void *basis,
                            unsigned *err, cudaStream_t st, int *launched);
// DFT_GEMM_F16X3: the per-frame scale of every frame of the batch into
// a.frame_scale (one warp per frame over the window's support).
cudaError_t launch_frame_scale(const FrontArgs &a, const DftShape &s, cudaStream_t st);

// Frame kernel: framing + window + rFFT + |X|^2 + mode epilogue.
cudaError_t launch_frontend(int log2n, int mode, int variant, const FrontArgs &a, int grid_limit,
                            cudaStream_t s, int *launched_grid);
cudaError_t launch_dct(const DctArgs &a, cudaStream_t s);
cudaError_t launch_fill_u32(unsigned *p, unsigned v, long long n, cudaStream_t s);
// Deterministic pseudo-random samples in [-0.5, 0.5) (autotuning inputs).
cudaError_t launch_fill_pattern(float *p, long long n, cudaStream_t s);

// dB scaling over a flat array: pass 1 writes mult*log10(max(x,amin)/ref) and the
// encoded max into *slot; pass 2 floors at max - top_db.
// ref_slot (2 words, optional): take the reference value as max(x) on the device.
cudaError_t launch_db(const float *x, float *y, long long n, float mult, float amin,
                      float ref, float top_db, unsigned *slot, cudaStream_t s,
                      unsigned *ref_slot = nullptr);
cudaError_t build_mel_dense(float *W, int4 *info, int sr, int n_fft, int n_mels, float fmin, float fmax,
                            cudaStream_t s);
cudaError_t build_dct_basis_rows(float *B, int n_out, int n_rows, cudaStream_t s);

unsigned encode_max_init();  // encoding of -inf
float decode_max(unsigned u);  // host-side inverse of the max encoding

}  // namespace mm
