// Plans (mm_plan_*): a fixed set of clips, their tables and device buffers
// kept resident, and their launches captured in a CUDA graph.  No
// counterpart in the reference, which re-plans every call (Bridge.swift:402).
//
// A plan is a list of sub-batches.  Clips are grouped by parameter set (first
// appearance order) and each group is cut into sub-batches of at most
// max_clips_per_branch clips.  Every sub-batch has its own layout (flattened
// frame index, persistent launches with the autotuned variant of its n_fft),
// its own region of the plan's single device allocation and its own branch
// stream.  The plan's graph forks the branches from one stream and joins them
// again, so sub-batches of different groups run concurrently; with host I/O
// (mm_plan_execute_host) each branch copies its own clips in and its results
// out, so one branch's copies overlap another branch's kernels.
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "runtime.h"

using namespace mm;

namespace {

constexpr int kSlots = 64;

struct Sub {
  Group g;
  Layout L;
  const DevTables *t = nullptr;
  DevBatch b;
  size_t arena_off = 0;   // bytes from the plan's base
  std::vector<int> clips;  // plan clip index of each local clip
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaEvent_t in_done = nullptr;  // execute_host: this sub-batch's inputs have landed
  cudaGraph_t graph = nullptr;  // this sub-batch's launches alone
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
};

struct Plan {
  std::vector<Sub> subs;
  std::vector<std::pair<int, int>> where;  // plan clip -> (sub, local clip)
  char *base = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;  // every sub-batch, forked and joined
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[kSlots][4] = {};
  int launches = 0;
  int device = 0;
};

void plan_free(Plan *p) {
  if (!p) return;
  if (p->stream) cudaStreamSynchronize(p->stream);
  for (Sub &s : p->subs) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.exec) cudaGraphExecDestroy(s.exec);
    if (s.graph) cudaGraphDestroy(s.graph);
    if (s.done) cudaEventDestroy(s.done);
    if (s.in_done) cudaEventDestroy(s.in_done);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  for (int s = 0; s < kSlots; s++)
    for (int q = 0; q < 4; q++)
      if (p->ev[s][q]) cudaEventDestroy(p->ev[s][q]);
  if (p->fork) cudaEventDestroy(p->fork);
  if (p->base) cudaFree(p->base);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

inline size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

Plan *plan_build(const std::vector<Group> &groups, const std::vector<int> &group_of, const int64_t *lengths,
                 int n_clips, int max_per_branch, int *status) {
  *status = MM_ERR_INVALID_INPUT;
  Plan *p = new (std::nothrow) Plan();
  if (!p) {
    *status = MM_ERR_ALLOC_FAILED;
    return nullptr;
  }
  cudaGetDevice(&p->device);
  p->where.assign(n_clips, {0, 0});
  // sub-batches: per group, clips in order, at most max_per_branch each
  for (size_t gi = 0; gi < groups.size(); gi++) {
    std::vector<int> members;
    for (int i = 0; i < n_clips; i++)
      if (group_of[i] == (int)gi) members.push_back(i);
    const int cap = max_per_branch > 0 ? max_per_branch : (int)members.size();
    for (size_t s0 = 0; s0 < members.size(); s0 += cap) {
      Sub s;
      s.g = groups[gi];
      s.g.variant = group_variant(s.g);
      s.clips.assign(members.begin() + s0, members.begin() + std::min(members.size(), s0 + cap));
      p->subs.push_back(std::move(s));
    }
  }
  int st = MM_OK;
  size_t total = 0;
  for (size_t si = 0; si < p->subs.size() && st == MM_OK; si++) {
    Sub &s = p->subs[si];
    s.t = get_tables(s.g, &st);
    if (!s.t) break;
    std::vector<int64_t> lens;
    for (size_t k = 0; k < s.clips.size(); k++) {
      lens.push_back(lengths[s.clips[k]]);
      p->where[s.clips[k]] = {(int)si, (int)k};
    }
    make_layout(s.g, lens.data(), (int)lens.size(), s.L);
    s.arena_off = total;
    total += up256(arena_bytes(s.g, s.L));
  }
  if (st != MM_OK) {
    *status = st;
    plan_free(p);
    return nullptr;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&p->base, total > 0 ? total : 256);
  for (Sub &s : p->subs) {
    if (e != cudaSuccess) break;
    e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.in_done, cudaEventDisableTiming);
    if (e != cudaSuccess) break;
    char *arena = p->base + s.arena_off;
    const size_t desc = carve_arena(s.g, s.L, arena, s.b);
    std::vector<char> host(desc + 16);
    pack_descriptors(s.L, host.data());
    e = cudaMemsetAsync(arena, 0, sizeof(float) * (size_t)s.L.sig_elems, p->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.b.clips, host.data(), desc, cudaMemcpyHostToDevice, p->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  }
  for (int q = 0; q < kSlots && e == cudaSuccess; q++)
    for (int r = 0; r < 4 && e == cudaSuccess; r++) e = cudaEventCreate(&p->ev[q][r]);
  // one graph per sub-batch (host I/O path) ...
  for (Sub &s : p->subs) {
    if (e != cudaSuccess) break;
    e = cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) break;
    cudaError_t e1 = enqueue_batch(s.g, s.L, s.t, s.b, s.stream, nullptr, &s.launches);
    cudaError_t e2 = cudaStreamEndCapture(s.stream, &s.graph);
    e = (e1 != cudaSuccess) ? e1 : e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&s.exec, s.graph, 0);
    p->launches += s.launches;
  }
  // ... and the whole plan: fork from p->stream, one branch per sub-batch, join
  if (e == cudaSuccess) e = cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    cudaError_t e1 = cudaEventRecord(p->fork, p->stream);
    for (Sub &s : p->subs) {
      if (e1 != cudaSuccess) break;
      e1 = cudaStreamWaitEvent(s.stream, p->fork, 0);
      if (e1 == cudaSuccess) e1 = enqueue_batch(s.g, s.L, s.t, s.b, s.stream, nullptr, nullptr);
      if (e1 == cudaSuccess) e1 = cudaEventRecord(s.done, s.stream);
      if (e1 == cudaSuccess) e1 = cudaStreamWaitEvent(p->stream, s.done, 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(p->stream, &p->graph);
    e = (e1 != cudaSuccess) ? e1 : e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *status = cuda_status(e);
    plan_free(p);
    return nullptr;
  }
  *status = MM_OK;
  return p;
}

Plan *as_plan(mm_plan h) { return static_cast<Plan *>(h); }

bool clip_ok(const Plan *p, int32_t clip) { return p && clip >= 0 && clip < (int)p->where.size(); }

}  // namespace

extern "C" {

mm_plan mm_plan_create(mm_context ctx, const MMFrontEndParams *params, const int64_t *lengths,
                       int32_t n_clips, int32_t *status) {
  int dummy;
  int32_t *st_out = status ? status : &dummy;
  *st_out = MM_ERR_INVALID_INPUT;
  if (!ctx || !lengths || n_clips <= 0) return nullptr;
  for (int i = 0; i < n_clips; i++)
    if (lengths[i] <= 0) return nullptr;
  Group g;
  int st = resolve_frontend(params, g);
  if (st == MM_OK) st = gpu_available();
  if (st != MM_OK) {
    *st_out = st;
    return nullptr;
  }
  std::vector<int> group_of(n_clips, 0);
  int s = MM_OK;
  Plan *p = plan_build({g}, group_of, lengths, n_clips, 0, &s);
  *st_out = s;
  return p;
}

mm_plan mm_plan_create_groups(mm_context ctx, const MMFrontEndParams *clip_params, const int64_t *lengths,
                              int32_t n_clips, int32_t max_clips_per_branch, int32_t *status) {
  int dummy;
  int32_t *st_out = status ? status : &dummy;
  *st_out = MM_ERR_INVALID_INPUT;
  if (!ctx || !clip_params || !lengths || n_clips <= 0 || max_clips_per_branch < 0) return nullptr;
  std::vector<Group> groups;
  std::vector<int> group_of(n_clips, 0);
  for (int i = 0; i < n_clips; i++) {
    if (lengths[i] <= 0) return nullptr;
    Group g;
    const int st = resolve_frontend(clip_params + i, g);
    if (st != MM_OK) {
      *st_out = st;
      return nullptr;
    }
    int k = 0;
    while (k < (int)groups.size() && !same_group(groups[k], g)) k++;
    if (k == (int)groups.size()) groups.push_back(g);
    group_of[i] = k;
  }
  const int st = gpu_available();
  if (st != MM_OK) {
    *st_out = st;
    return nullptr;
  }
  int s = MM_OK;
  Plan *p = plan_build(groups, group_of, lengths, n_clips, max_clips_per_branch, &s);
  *st_out = s;
  return p;
}

void mm_plan_destroy(mm_plan plan) { plan_free(as_plan(plan)); }

float *mm_plan_device_input(mm_plan plan) {
  return plan ? reinterpret_cast<float *>(as_plan(plan)->base) : nullptr;
}
float *mm_plan_device_output(mm_plan plan) {
  return plan ? reinterpret_cast<float *>(as_plan(plan)->base) : nullptr;
}

int64_t mm_plan_input_offset(mm_plan plan, int32_t clip) {
  Plan *p = as_plan(plan);
  if (!clip_ok(p, clip)) return -1;
  const Sub &s = p->subs[p->where[clip].first];
  return (int64_t)((reinterpret_cast<char *>(s.b.signal) - p->base) / sizeof(float)) +
         s.L.clips[p->where[clip].second].sig_off;
}
int64_t mm_plan_output_offset(mm_plan plan, int32_t clip) {
  Plan *p = as_plan(plan);
  if (!clip_ok(p, clip)) return -1;
  const Sub &s = p->subs[p->where[clip].first];
  return (int64_t)((reinterpret_cast<char *>(s.b.out) - p->base) / sizeof(float)) +
         s.L.clips[p->where[clip].second].out_off;
}
int64_t mm_plan_clip_frames(mm_plan plan, int32_t clip) {
  Plan *p = as_plan(plan);
  if (!clip_ok(p, clip)) return -1;
  return p->subs[p->where[clip].first].L.clips[p->where[clip].second].n_frames;
}
int32_t mm_plan_clip_rows(mm_plan plan, int32_t clip) {
  Plan *p = as_plan(plan);
  if (!clip_ok(p, clip)) return -1;
  return output_rows(p->subs[p->where[clip].first].g);
}
int32_t mm_plan_rows(mm_plan plan) {
  Plan *p = as_plan(plan);
  if (!p || p->subs.empty()) return -1;
  const int r = output_rows(p->subs[0].g);
  for (const Sub &s : p->subs)
    if (output_rows(s.g) != r) return -1;
  return r;
}
int64_t mm_plan_total_frames(mm_plan plan) {
  Plan *p = as_plan(plan);
  if (!p) return -1;
  int64_t t = 0;
  for (const Sub &s : p->subs) t += s.L.total_frames;
  return t;
}
int32_t mm_plan_kernel_launches(mm_plan plan) { return plan ? as_plan(plan)->launches : -1; }
int32_t mm_plan_branches(mm_plan plan) { return plan ? (int32_t)as_plan(plan)->subs.size() : -1; }

float *mm_plan_device_mel_db(mm_plan plan) {
  Plan *p = as_plan(plan);
  return (p && p->subs.size() == 1) ? p->subs[0].b.meldb : nullptr;
}

const float *mm_plan_clip_mel_db(mm_plan plan, int32_t clip) {
  Plan *p = as_plan(plan);
  if (!clip_ok(p, clip)) return nullptr;
  const Sub &s = p->subs[p->where[clip].first];
  if (s.g.mode != MODE_MELDB || !s.b.meldb) return nullptr;
  return s.b.meldb + s.L.clips[p->where[clip].second].frame_off * (long long)s.g.n_mels;
}

int32_t mm_plan_clip_max_db(mm_plan plan, int32_t clip, float *max_db) {
  Plan *p = as_plan(plan);
  if (!clip_ok(p, clip) || !max_db) return MM_ERR_INVALID_INPUT;
  const Sub &s = p->subs[p->where[clip].first];
  unsigned u = 0;
  cudaError_t e = cudaMemcpy(&u, s.b.clip_max + p->where[clip].second, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  *max_db = decode_max(u);
  return MM_OK;
}

int32_t mm_plan_execute(mm_plan plan, void *stream) {
  Plan *p = as_plan(plan);
  if (!p) return MM_ERR_INVALID_INPUT;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
  return cuda_status(cudaGraphLaunch(p->exec, s));
}

int32_t mm_plan_execute_timed(mm_plan plan, void *stream, int32_t slot) {
  Plan *p = as_plan(plan);
  if (!p || slot < 0 || slot >= kSlots || p->subs.size() != 1) return MM_ERR_INVALID_INPUT;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
  const Sub &b = p->subs[0];
  return cuda_status(enqueue_batch(b.g, b.L, b.t, b.b, s, p->ev[slot], nullptr));
}

int32_t mm_plan_stage_ms(mm_plan plan, int32_t slot, float *ms3) {
  Plan *p = as_plan(plan);
  if (!p || slot < 0 || slot >= kSlots || !ms3) return MM_ERR_INVALID_INPUT;
  for (int q = 0; q < 3; q++) {
    cudaError_t e = cudaEventElapsedTime(&ms3[q], p->ev[slot][q], p->ev[slot][q + 1]);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return MM_OK;
}

int32_t mm_plan_execute_host(mm_plan plan, const float *const *signals, float *const *outs, void *stream) {
  Plan *p = as_plan(plan);
  if (!p || !signals || !outs) return MM_ERR_INVALID_INPUT;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : p->stream;
  cudaError_t e = cudaEventRecord(p->fork, s);
  // The uploads are chained in branch order (each branch's copies start when
  // the previous branch's have landed), so the host link carries one branch
  // at a time and branch i's kernels run while branch i+1 uploads; issued
  // side by side, the branches would share the link and land together.
  cudaEvent_t prev = p->fork;
  for (Sub &b : p->subs) {
    if (e != cudaSuccess) break;
    e = cudaStreamWaitEvent(b.stream, prev, 0);
    // one copy per run of clips whose host buffers follow each other and whose
    // device slots do too (e.g. the rows of one [n, length] host array): each
    // copy carries a fixed cost, so hundreds of per-clip copies cost link time
    const size_t n = b.clips.size();
    for (size_t k = 0; k < n && e == cudaSuccess;) {
      const ClipDesc &c = b.L.clips[k];
      const float *h = signals[b.clips[k]];
      size_t len = (size_t)c.length, j = k + 1;
      while (j < n && signals[b.clips[j]] == h + len && b.L.clips[j].sig_off == c.sig_off + (long long)len) {
        len += (size_t)b.L.clips[j].length;
        j++;
      }
      e = cudaMemcpyAsync(b.b.signal + c.sig_off, h, sizeof(float) * len, cudaMemcpyHostToDevice, b.stream);
      k = j;
    }
    if (e == cudaSuccess) e = cudaEventRecord(b.in_done, b.stream);
    prev = b.in_done;
    if (e == cudaSuccess) e = cudaGraphLaunch(b.exec, b.stream);
    const int rows = output_rows(b.g);
    for (size_t k = 0; k < n && e == cudaSuccess;) {
      const ClipDesc &c = b.L.clips[k];
      float *h = outs[b.clips[k]];
      size_t cnt = (size_t)rows * (size_t)c.n_frames, j = k + 1;
      while (j < n && outs[b.clips[j]] == h + cnt && b.L.clips[j].out_off == c.out_off + (long long)cnt) {
        cnt += (size_t)rows * (size_t)b.L.clips[j].n_frames;
        j++;
      }
      if (cnt)
        e = cudaMemcpyAsync(h, b.b.out + c.out_off, sizeof(float) * cnt, cudaMemcpyDeviceToHost, b.stream);
      k = j;
    }
    if (e == cudaSuccess) e = cudaEventRecord(b.done, b.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b.done, 0);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e);
  for (const Sub &b : p->subs) {
    const int st = take_error_word(b.g, b.t);
    if (st != MM_OK) return st;
  }
  return MM_OK;
}

int32_t mm_plan_status(mm_plan plan, void *stream) {
  Plan *p = as_plan(plan);
  if (!p) return MM_ERR_INVALID_INPUT;
  cudaError_t e = cudaStreamSynchronize(stream ? static_cast<cudaStream_t>(stream) : p->stream);
  if (e != cudaSuccess) return cuda_status(e);
  for (const Sub &b : p->subs) {
    const int st = take_error_word(b.g, b.t);
    if (st != MM_OK) return st;
  }
  return MM_OK;
}

}  // extern "C"
