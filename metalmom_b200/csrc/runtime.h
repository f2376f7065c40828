// Host runtime of libmetalmom.so: device checks, resident tables, batch
// layout, per-thread workspaces and the launch sequence of one batch.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "kernels.h"
#include "metalmom.h"

namespace mm {

// Map a CUDA error to an MM_ERR_* status.
int cuda_status(cudaError_t e);
// MM_OK when a CUDA device is usable, else MM_ERR_METAL_UNAVAILABLE.
int gpu_available();

// Fully resolved parameters of one group (reference sentinels applied).
struct Group {
  int mode = MODE_MELDB;
  int sr = 22050, n_fft = 2048, log2n = 11, hop = 512, win = 2048;
  int center = 1, pad_mode = PAD_CONSTANT, window_zero = 0;
  int n_mels = 128, n_mfcc_eff = 20;
  float fmin = 0.0f, fmax = 11025.0f, top_db = 80.0f;
  float power = 2.0f, amin = 1e-10f, ref = 1.0f;
  int variant = 0;  // frame-kernel launch variant (autotuned per n_fft)
  int dft_form = DFT_FFT_F32;
  int post = POST_DCT;  // MODE_MELDB: DCT (MFCC) or onset strength
  int lag = 1;          // onset difference lag
};

// Process-wide autotuning table: launch variant per log2(n_fft).
int tuned_variant(int log2n);
void set_tuned_variant(int log2n, int v);
// The variant a group of this mode/power/size runs with (0 when not tunable).
int group_variant(const Group &g);

int is_pow2(long long n);
int ilog2(long long n);
// Reference frame count (STFT.swift:241-262): 0 when padded < n_fft or n_fft
// is not a power of two.
long long frame_count(long long length, int n_fft, int hop, int center);
// Rows of one clip's output block for the group's mode.
int output_rows(const Group &g);

// True when two groups launch identically (clips of both can share a batch).
bool same_group(const Group &a, const Group &b);

// MFCC-path group from MMFrontEndParams (sentinels of mm_mfcc, pad mode,
// top_db); MM_ERR_INVALID_INPUT for unsupported values.
int resolve_frontend(const MMFrontEndParams *p, Group &g);

// Resident tables for (device, sr, n_fft, win, n_mels, fmin, fmax, n_mfcc).
const DevTables *get_tables(const Group &g, int *status);

struct Layout {
  std::vector<ClipDesc> clips;
  std::vector<int> tile_clip;       // frame tiles
  std::vector<int> dct_tile_clip;   // DCT tiles
  std::vector<int> dct_tile_first;
  long long sig_elems = 0, total_frames = 0, out_elems = 0, meldb_elems = 0;
  long long scale_elems = 0;  // per-frame scales (fp16-split DFT form only)
  int F = 1;
};
void make_layout(const Group &g, const int64_t *lengths, int n, Layout &L);

// Device-side pointers of one batch.
struct DevBatch {
  float *signal = nullptr;
  ClipDesc *clips = nullptr;
  int *tile_clip = nullptr;
  int *dct_tile_clip = nullptr;
  int *dct_tile_first = nullptr;
  unsigned *clip_max = nullptr;
  float *meldb = nullptr;
  float *out = nullptr;
  float *frame_scale = nullptr;
};

// Bytes of one device arena holding a whole batch (signal included).
size_t arena_bytes(const Group &g, const Layout &L);
// Carve the arena into DevBatch pointers; returns the bytes of the
// descriptor region (clips + tile tables) that starts at ->clips.
size_t carve_arena(const Group &g, const Layout &L, char *base, DevBatch &b);
// Serialise the descriptor region (same order as carve_arena) into host memory.
void pack_descriptors(const Layout &L, char *host);

// Enqueue the launch sequence of one batch.  `ev` may be null or point to 4
// events recorded before/after the stages (frame kernel, DCT).
// After the group's work has completed on the device: MM_ERR_INTERNAL (and
// the word cleared) when a bounded wait of one of its tensor-core kernels ran
// out, else MM_OK.  Reads the error word only for groups that launch such
// kernels (the DFT-as-GEMM forms, the tensor-core frame kernel).
int take_error_word(const Group &g, const DevTables *t);

cudaError_t enqueue_batch(const Group &g, const Layout &L, const DevTables *t, const DevBatch &b,
                          cudaStream_t s, cudaEvent_t *ev, int *n_launches);

// Per-thread scratch: a stream, a growable device arena and pinned staging.
struct Workspace {
  int device = -1;
  cudaStream_t stream = nullptr;
  char *dev = nullptr;
  size_t dev_bytes = 0;
  char *host = nullptr;
  size_t host_bytes = 0;
};
// Returns the calling thread's workspace with at least the requested sizes.
int thread_workspace(size_t dev_bytes, size_t host_bytes, Workspace **ws);

// Fill an MMBuffer with a 2-D shape; data may be null when count is 0.
void fill_buffer(MMBuffer *out, float *data, long long rows, long long cols);

}  // namespace mm
