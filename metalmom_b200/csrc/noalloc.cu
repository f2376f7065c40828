// mm_mfcc_noalloc: MFCC of one clip already on the device, with every piece of
// scratch memory taken from a fixed array compiled into the library.
//
// Who needs this: callers that must not allocate device memory while they
// run -- code running inside another framework's memory pool or under a
// strict memory budget, real-time audio threads that may not block in the
// allocator, and plugin hosts that hand in device buffers but forbid
// cudaMalloc/cudaFree.  They pass the signal and the output buffer; the
// filterbank, DCT basis, twiddles, frame tables and the log-mel scratch all
// live in `g_noalloc_scratch` below.
//
// The array holds kNoallocScratchBytes (16 MiB) on every GPU that loads the
// library, for as long as the library stays loaded.  Every call shares it and
// it keeps the previous call's contents: the tables of the last parameter set
// stay at its start, and the per-clip maximum is reset on each call.  Two
// calls whose work overlaps on the GPU (different streams, or different host
// threads) race on the array.
//
// Cost per call: the first call with a parameter set (per device) builds the
// tables into the array and waits once on `stream` for the filterbank size;
// a call with the same parameters as the device's previous call enqueues one
// descriptor kernel, the frame kernel and the DCT, and does not wait.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "runtime.h"

namespace {

constexpr size_t kNoallocScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// What the array's start holds on one device: the tables of one parameter set.
struct TableKey {
  int sr = 0, n_fft = 0, win = 0, n_mels = 0, n_mfcc_eff = 0;
  float fmin = 0.0f, fmax = 0.0f;
  bool operator==(const TableKey &o) const {
    return sr == o.sr && n_fft == o.n_fft && win == o.win && n_mels == o.n_mels && n_mfcc_eff == o.n_mfcc_eff &&
           fmin == o.fmin && fmax == o.fmax;
  }
};

struct DeviceState {
  void *base = nullptr;  // device address of the array (looked up once)
  bool built = false;
  TableKey key;
  mm::DevTables t;
  size_t used = 0;  // bytes of the array the tables take (256-byte multiple)
};

std::mutex g_noalloc_mu;
DeviceState g_noalloc_dev[kMaxDevices];

// Device address of the scratch array for the current device.  The host-side
// name `g_noalloc_scratch` is only a stand-in: the address is looked up once
// per device, at that device's first call, with the device current.  (A
// device reset unloads the module; calls after one are not supported.)  The
// caller holds g_noalloc_mu.
int noalloc_scratch(int dev, char **out) {
  DeviceState &d = g_noalloc_dev[dev];
  if (!d.base) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return MM_ERR_INTERNAL;
    }
    d.base = p;
    d.built = false;
  }
  *out = static_cast<char *>(d.base);
  return MM_OK;
}

// Single-clip descriptors and the reset clip maximum, written on the device
// (no host copies).
__global__ void noalloc_desc_kernel(mm::ClipDesc *cd, long long sig_off, long long length, int n_frames,
                                    int *tile_clip, int tiles, int *dct_clip, int *dct_first, int dct_tiles,
                                    unsigned *clip_max, unsigned max_init) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    cd->sig_off = sig_off;
    cd->length = length;
    cd->frame_off = 0;
    cd->out_off = 0;
    cd->n_frames = n_frames;
    cd->tile_base = 0;
    *clip_max = max_init;
  }
  for (int k = i; k < tiles; k += gridDim.x * blockDim.x) tile_clip[k] = 0;
  for (int k = i; k < dct_tiles; k += gridDim.x * blockDim.x) {
    dct_clip[k] = 0;
    dct_first[k] = k * mm::kDctTile;
  }
}

inline size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" MM_API int32_t mm_mfcc_noalloc(const float *d_signal, int64_t signal_length, int32_t sample_rate,
                                          int32_t n_mfcc, int32_t n_fft, int32_t hop_length,
                                          int32_t win_length, int32_t n_mels, float f_min, float f_max,
                                          int32_t center, float *d_out, void *stream) {
  using namespace mm;
  if (!d_signal || signal_length <= 0 || !d_out) return MM_ERR_INVALID_INPUT;
  if ((reinterpret_cast<uintptr_t>(d_signal) & 3) != 0) return MM_ERR_INVALID_INPUT;
  if (n_fft <= 0 || n_mels < 0 || n_mfcc < 0) return MM_ERR_INVALID_INPUT;
  Group g;
  g.mode = MODE_MELDB;
  g.sr = sample_rate;
  g.n_fft = n_fft;
  g.log2n = ilog2(n_fft);
  g.hop = hop_length > 0 ? hop_length : n_fft / 4;
  g.win = win_length > 0 ? win_length : n_fft;
  g.center = center != 0;
  g.pad_mode = PAD_CONSTANT;
  g.n_mels = n_mels;
  g.n_mfcc_eff = std::min(n_mfcc, n_mels);
  g.fmin = f_min;
  g.fmax = f_max > 0.0f ? f_max : (float)sample_rate / 2.0f;
  g.power = 2.0f;
  g.amin = 1e-10f;
  g.ref = 1.0f;
  g.top_db = 80.0f;
  if (g.hop <= 0) return MM_ERR_INVALID_INPUT;
  const long long T = frame_count(signal_length, g.n_fft, g.hop, g.center);
  if (T == 0 || g.n_mfcc_eff == 0) return MM_OK;  // empty result: nothing to write
  if (g.log2n > 15) return MM_ERR_INVALID_INPUT;
  int st = gpu_available();
  if (st != MM_OK) return st;
  g.variant = group_variant(g);
  if (g.variant == kTcVariant) g.variant = kWarpVariant;  // its bounded waits report to a table's error word

  // Scratch needed beyond the tables: descriptors, clip max, log-mel rows.
  const int F = frames_per_tile(g.log2n, g.variant);
  const int tiles = (int)((T + F - 1) / F);
  const int dct_tiles = (int)((T + kDctTile - 1) / kDctTile);
  const size_t batch_bytes = up256(sizeof(ClipDesc)) + up256(sizeof(int) * (size_t)tiles) +
                             2 * up256(sizeof(int) * (size_t)dct_tiles) + up256(sizeof(unsigned)) +
                             up256(sizeof(float) * (size_t)T * (size_t)n_mels);
  if (batch_bytes >= kNoallocScratchBytes) return MM_ERR_INVALID_INPUT;  // clip too long for the scratch

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= kMaxDevices) return MM_ERR_INTERNAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TableKey key;
  key.sr = g.sr;
  key.n_fft = g.n_fft;
  key.win = g.win;
  key.n_mels = g.n_mels;
  key.n_mfcc_eff = g.n_mfcc_eff;
  key.fmin = g.fmin;
  key.fmax = g.fmax;

  char *base = nullptr;
  DevTables t;
  size_t used = 0;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if ((st = noalloc_scratch(dev, &base)) != MM_OK) return st;
    DeviceState &d = g_noalloc_dev[dev];
    if (!(d.built && d.key == key)) {
      // (Re)build this parameter set's tables at the array's start; the
      // previous set's tables are gone from here on.
      d.built = false;
      e = build_tables_at(d.t, base, kNoallocScratchBytes, &d.used, g.sr, g.n_fft, g.win, g.n_mels, g.fmin,
                          g.fmax, g.n_mfcc_eff, 0, s);
      if (e == cudaErrorMemoryAllocation) return MM_ERR_INVALID_INPUT;  // tables too large for the scratch
      if (e != cudaSuccess) return cuda_status(e);
      d.key = key;
      d.built = true;
    }
    t = d.t;
    used = d.used;
  }
  if (used + batch_bytes > kNoallocScratchBytes) return MM_ERR_INVALID_INPUT;  // clip too long for the scratch

  char *p = base + used;
  ClipDesc *cd = reinterpret_cast<ClipDesc *>(p);
  p += up256(sizeof(ClipDesc));
  int *tile_clip = reinterpret_cast<int *>(p);
  p += up256(sizeof(int) * (size_t)tiles);
  int *dct_clip = reinterpret_cast<int *>(p);
  p += up256(sizeof(int) * (size_t)dct_tiles);
  int *dct_first = reinterpret_cast<int *>(p);
  p += up256(sizeof(int) * (size_t)dct_tiles);
  unsigned *clip_max = reinterpret_cast<unsigned *>(p);
  p += up256(sizeof(unsigned));
  float *meldb = reinterpret_cast<float *>(p);

  // The frame kernel reads float2 pairs relative to an 8-byte aligned base:
  // address a 4-byte aligned signal as base + 1.
  const long long sig_off = (long long)((reinterpret_cast<uintptr_t>(d_signal) & 7) / 4);
  const float *sig_base = d_signal - sig_off;

  const int nb = std::max(1, std::min(1024, (std::max(tiles, dct_tiles) + 255) / 256));
  noalloc_desc_kernel<<<nb, 256, 0, s>>>(cd, sig_off, signal_length, (int)T, tile_clip, tiles, dct_clip,
                                         dct_first, dct_tiles, clip_max, encode_max_init());
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e);

  FrontArgs a;
  a.signal = sig_base;
  a.clips = cd;
  a.tile_clip = tile_clip;
  a.total_tiles = tiles;
  a.hop = g.hop;
  a.pad = g.center ? g.n_fft / 2 : 0;
  a.pad_mode = g.pad_mode;
  a.window = t.window;
  a.tw_stage = t.tw_stage;
  a.tw_split = t.tw_split;
  a.tw_tiny = t.tw_tiny;
  a.mel_info = t.mel_info;
  a.mel_pw = t.mel_pw;
  a.mel_nnz = t.mel_nnz;
  a.mel_w2 = t.mel_w2;
  a.mel_seg = t.mel_seg;
  a.mel_seg_ok = t.mel_seg_ok;
  a.mel_lw = t.mel_lw;
  a.mel_lane = t.mel_lane;
  a.mel_band = t.mel_band;
  a.mel_lane_ok = t.mel_lane_ok;
  a.n_mels = g.n_mels;
  a.power = 2.0f;
  a.amin = g.amin;
  a.ref = g.ref;
  a.out = meldb;
  a.clip_max = clip_max;
  if ((e = launch_frontend(g.log2n, MODE_MELDB, g.variant, a, 0, s, nullptr)) != cudaSuccess)
    return cuda_status(e);

  DctArgs d;
  d.mel_db = meldb;
  d.clips = cd;
  d.tile_clip = dct_clip;
  d.tile_first = dct_first;
  d.total_tiles = dct_tiles;
  d.clip_max = clip_max;
  d.basis = t.dct;
  d.n_mels = g.n_mels;
  d.n_mfcc = g.n_mfcc_eff;
  d.top_db = g.top_db;
  d.out = d_out;
  if ((e = launch_dct(d, s)) != cudaSuccess) return cuda_status(e);
  return MM_OK;
}
