// Serving engine of libmetalmom.so (mm_server_*): continuous batching of MFCC
// requests with device-memory admission.  No counterpart in the reference,
// which computes one clip per call (Bridge.swift:402 mm_mfcc).
//
// One scheduler thread per server:
//   * submit() copies the request's samples into a pinned block from the
//     server's pinned pool (the only host copy of the samples) and queues it;
//   * whenever one of `max_inflight` stream slots is free, the scheduler
//     takes the oldest pending request and every other pending request of
//     the same parameter group (FIFO, up to max_batch_clips and the free part
//     of the device budget) and enqueues H2D of each pinned block -> frame
//     kernel -> DCT -> D2H on the slot's stream, with a stream-ordered device
//     arena (cudaMallocAsync);
//   * a host callback at the end of the stream marks the batch finished; the
//     scheduler then hands each request its result, releases the arena and
//     the budget, and refills the slot with whatever arrived meanwhile.
// Requests that arrive while batches run are therefore admitted as slots and
// memory free up, and batches of different groups run concurrently.
// Filterbanks and other tables stay resident per group (get_tables).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "runtime.h"

using namespace mm;

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { REQ_PENDING = 0, REQ_RUNNING = 1, REQ_DONE = 2, REQ_FAILED = 3 };

// Pinned host blocks in power-of-two size classes, carved from 256 MiB chunks
// that stay allocated until the server is destroyed (freeing pinned memory
// would synchronise the device).  get() returns null when the pinned total
// would exceed the cap; the request then keeps a pageable copy.
class PinnedPool {
 public:
  static constexpr size_t kChunk = size_t(256) << 20;
  explicit PinnedPool(size_t cap) : cap_(cap) {}
  ~PinnedPool() {
    for (char *c : chunks_) cudaFreeHost(c);
  }
  static int size_class(size_t bytes) {
    int c = 12;
    while ((size_t(1) << c) < bytes) c++;
    return c;
  }
  // Pins `bytes` (whole chunks, within the cap) up front, so that serving
  // does not stop in cudaMallocHost (tens of milliseconds per chunk, under a
  // driver lock that the scheduler's launches wait on) until that is used up.
  cudaError_t reserve(size_t bytes) {
    std::lock_guard<std::mutex> lk(mu_);
    while (spare_.size() * kChunk < bytes && total_ + kChunk <= cap_) {
      char *p = nullptr;
      cudaError_t e = cudaMallocHost(&p, kChunk);
      if (e != cudaSuccess) return e;
      chunks_.push_back(p);
      spare_.push_back(p);
      total_ += kChunk;
    }
    return cudaSuccess;
  }
  float *get(size_t bytes, int *cls) {
    const int c = size_class(bytes);
    const size_t sz = size_t(1) << c;
    std::lock_guard<std::mutex> lk(mu_);
    *cls = c;
    if (!free_[c].empty()) {
      char *p = free_[c].back();
      free_[c].pop_back();
      return reinterpret_cast<float *>(p);
    }
    if (sz > kChunk) {  // a block of its own
      if (total_ + sz > cap_) return nullptr;
      char *p = nullptr;
      if (cudaMallocHost(&p, sz) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
      chunks_.push_back(p);
      total_ += sz;
      return reinterpret_cast<float *>(p);
    }
    if (left_ < sz) {
      char *p = nullptr;
      if (!spare_.empty()) {  // a chunk pinned at creation
        p = spare_.back();
        spare_.pop_back();
      } else {
        if (total_ + kChunk > cap_) return nullptr;
        if (cudaMallocHost(&p, kChunk) != cudaSuccess) {
          cudaGetLastError();
          return nullptr;
        }
        chunks_.push_back(p);
        total_ += kChunk;
      }
      cur_ = p;
      left_ = kChunk;
    }
    char *p = cur_;
    cur_ += sz;
    left_ -= sz;
    return reinterpret_cast<float *>(p);
  }
  void put(float *p, int cls) {
    std::lock_guard<std::mutex> lk(mu_);
    free_[cls].push_back(reinterpret_cast<char *>(p));
  }

 private:
  std::mutex mu_;
  std::vector<char *> chunks_;
  std::vector<char *> spare_;  // reserved chunks not carved yet
  std::vector<char *> free_[64];
  char *cur_ = nullptr;
  size_t left_ = 0, total_ = 0, cap_;

 public:
  size_t cap() const { return cap_; }
};

// A batch's results in one pinned block from the pool: the device copies
// them there, and each request's caller copies its own part out (outside the
// server lock) and drops a reference; the last one returns the block.  The
// scheduler thread then never copies results.
struct ResultBlock {
  float *data = nullptr;
  int cls = 0;
  std::atomic<int> refs{0};
};

struct Request {
  int64_t id = 0;
  Group g;
  long long length = 0;
  float *pin = nullptr;      // samples in a pinned block (pin_cls = its size class) ...
  int pin_cls = 0;
  std::vector<float> signal;  // ... or, when the pinned pool is full, a pageable copy ...
  const float *borrowed = nullptr;  // ... or the caller's own buffer (mm_server_submit_borrowed)
  float *result = nullptr;  // malloc'd [rows x frames], handed to the caller ...
  ResultBlock *block = nullptr;  // ... or its part of the batch's result block, copied out by the caller
  const float *block_src = nullptr;
  long long rows = 0, frames = 0;
  int state = REQ_PENDING;
  int status = MM_OK;
  Clock::time_point t_submit, t_done;
};

struct Server;

struct Slot {
  Server *srv = nullptr;
  cudaStream_t stream = nullptr;
  char *pinned = nullptr;
  size_t pinned_bytes = 0;
  // staging outgrown while serving: freed at destroy (cudaFreeHost would
  // synchronise the device in the middle of other batches)
  std::vector<char *> retired;
  // current batch
  bool busy = false;
  std::atomic<bool> finished{false};
  std::vector<Request *> reqs;
  Group g;
  Layout L;
  char *arena = nullptr;
  size_t arena_size = 0;
  size_t sig_bytes = 0, desc_bytes = 0, out_bytes = 0;
  ResultBlock *rblock = nullptr;  // this batch's results (else they land in `pinned`)
  int error = MM_OK;
};

struct Server {
  int device = 0;
  size_t budget = 0;
  PinnedPool *pool = nullptr;
  cudaMemPool_t mempool = nullptr;  // device arenas; keeps freed memory for reuse
  int max_batch = 256;
  std::vector<Slot *> slots;

  std::mutex mu;
  std::condition_variable cv;       // wakes the scheduler
  std::condition_variable done_cv;  // wakes waiters
  std::deque<Request *> pending;
  std::unordered_map<int64_t, Request *> reqs;
  int64_t next_id = 1;
  bool stop = false;
  std::thread worker;

  // accounting (under mu)
  size_t in_use = 0, peak = 0;
  int64_t submitted = 0, completed = 0, failed = 0, batches = 0;
  double audio_s = 0.0;
  double launch_ms = 0.0, finish_ms = 0.0;  // scheduler host time per phase
  std::vector<double> lat_ms;

  size_t pool_cap() const { return pool->cap(); }
  void run();
  bool admit_one(std::unique_lock<std::mutex> &lk);
  void finish(Slot *s);
};

void CUDART_CB on_stream_done(void *p) {
  Slot *s = static_cast<Slot *>(p);
  Server *srv = s->srv;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    s->finished.store(true);
  }
  srv->cv.notify_all();
}

// Take the next batch out of `pending` and launch it on a free slot.
// Returns false when nothing could be launched (no slot, nothing pending,
// or the head of the queue waits for memory).  Called with mu held; drops it
// while copying and enqueueing.
bool Server::admit_one(std::unique_lock<std::mutex> &lk) {
  Slot *slot = nullptr;
  for (Slot *s : slots)
    if (!s->busy) {
      slot = s;
      break;
    }
  if (!slot || pending.empty()) return false;

  Request *head = pending.front();
  const Group g0 = head->g;
  // FIFO scan: the head and the following requests of its group, while the
  // batch's arena fits in the free budget.
  std::vector<Request *> take;
  std::vector<int64_t> lens;
  Group g = g0;
  g.variant = group_variant(g);
  // per-clip upper bound of the arena (segments are 256-byte aligned)
  const int F = frames_per_tile(g.log2n, g.variant);
  const int rows = output_rows(g);
  size_t bytes = 8 * 256;
  for (Request *r : pending) {
    if ((int)take.size() >= max_batch) break;
    if (!same_group(r->g, g0)) continue;
    const long long T = frame_count(r->length, g.n_fft, g.hop, g.center);
    const size_t need = sizeof(float) * (size_t)((r->length + 3) / 4 * 4) + sizeof(ClipDesc) + 16 +
                        sizeof(int) * (size_t)((T + F - 1) / F) + 2 * sizeof(int) * (size_t)((T + kDctTile - 1) / kDctTile) +
                        sizeof(unsigned) + sizeof(float) * (size_t)T * (size_t)(g.n_mels + rows);
    if (in_use + bytes + need > budget) break;
    take.push_back(r);
    lens.push_back((int64_t)r->length);
    bytes += need;
  }
  Layout L;
  if (!take.empty()) {
    make_layout(g, lens.data(), (int)lens.size(), L);
    bytes = std::max(bytes, arena_bytes(g, L));
  }
  if (take.empty()) {
    bool any_busy = false;
    for (Slot *s : slots) any_busy |= s->busy;
    if (any_busy) return false;  // wait for memory to free up
    // nothing runs and the request alone exceeds the budget: it can never run
    pending.pop_front();
    head->state = REQ_FAILED;
    head->status = MM_ERR_ALLOC_FAILED;
    head->t_done = Clock::now();
    failed++;
    done_cv.notify_all();
    return true;
  }
  for (Request *r : take) {
    r->state = REQ_RUNNING;
    pending.erase(std::find(pending.begin(), pending.end(), r));
  }
  slot->busy = true;
  slot->finished.store(false);
  slot->reqs = take;
  slot->g = g;
  slot->L = std::move(L);
  slot->arena_size = bytes;
  slot->error = MM_OK;
  in_use += bytes;
  peak = std::max(peak, in_use);
  batches++;

  // ---- outside the lock: the launch sequence
  lk.unlock();
  const auto t_launch = Clock::now();
  int st = MM_OK;
  const DevTables *t = get_tables(g, &st);
  cudaError_t e = cudaSuccess;
  if (st == MM_OK) {
    DevBatch probe;
    slot->desc_bytes = carve_arena(g, slot->L, nullptr, probe);
    slot->sig_bytes = sizeof(float) * (size_t)slot->L.sig_elems;
    slot->out_bytes = sizeof(float) * (size_t)slot->L.out_elems;
    const size_t host_need = std::max(slot->desc_bytes, slot->out_bytes) + 256;
    if (host_need > slot->pinned_bytes) {
      const size_t grow = std::max(host_need + host_need / 4, 2 * slot->pinned_bytes);
      char *p = nullptr;
      e = cudaMallocHost(&p, grow);
      if (e == cudaSuccess) {
        if (slot->pinned) slot->retired.push_back(slot->pinned);
        slot->pinned = p;
        slot->pinned_bytes = grow;
      }
    }
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&slot->arena, bytes, mempool, slot->stream);
    if (e == cudaSuccess) {
      char *h = slot->pinned;
      pack_descriptors(slot->L, h);
      DevBatch b;
      carve_arena(g, slot->L, slot->arena, b);
      for (size_t i = 0; i < take.size() && e == cudaSuccess; i++) {
        const float *src = take[i]->pin ? take[i]->pin
                           : take[i]->borrowed ? take[i]->borrowed : take[i]->signal.data();
        e = cudaMemcpyAsync(b.signal + slot->L.clips[i].sig_off, src, sizeof(float) * (size_t)take[i]->length,
                            cudaMemcpyHostToDevice, slot->stream);
      }
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(b.clips, h, slot->desc_bytes, cudaMemcpyHostToDevice, slot->stream);
      if (e == cudaSuccess) e = enqueue_batch(g, slot->L, t, b, slot->stream, nullptr, nullptr);
      float *dst = reinterpret_cast<float *>(h);
      int rcls = 0;
      float *rb = pool->get(slot->out_bytes, &rcls);
      if (rb) {
        slot->rblock = new (std::nothrow) ResultBlock();
        if (slot->rblock) {
          slot->rblock->data = rb;
          slot->rblock->cls = rcls;
          dst = rb;
        } else {
          pool->put(rb, rcls);
        }
      }
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(dst, b.out, slot->out_bytes, cudaMemcpyDeviceToHost, slot->stream);
    }
    if (e != cudaSuccess) st = cuda_status(e);
  }
  if (st != MM_OK) {
    cudaGetLastError();
    slot->error = st;
  }
  // The callback also runs after a failed enqueue so that the batch is reaped.
  e = cudaLaunchHostFunc(slot->stream, on_stream_done, slot);
  const double dt = std::chrono::duration<double, std::milli>(Clock::now() - t_launch).count();
  lk.lock();
  launch_ms += dt;
  if (e != cudaSuccess) {
    cudaGetLastError();
    slot->error = cuda_status(e);
    slot->finished.store(true);
  }
  return true;
}

// Hand out the results of a finished batch (called with mu held).
void Server::finish(Slot *s) {
  const auto now = Clock::now();
  struct Timer {
    double *acc;
    Clock::time_point t0 = Clock::now();
    ~Timer() { *acc += std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
  } timer{&finish_ms};
  if (s->error == MM_OK) {  // a bounded wait of a tensor-core kernel of this batch ran out
    int dev_st = MM_OK;
    const DevTables *t = get_tables(s->g, &dev_st);
    if (t) s->error = take_error_word(s->g, t);
  }
  const int rows = output_rows(s->g);
  for (size_t i = 0; i < s->reqs.size(); i++) {
    Request *r = s->reqs[i];
    r->t_done = now;
    r->rows = rows;
    r->frames = s->L.clips[i].n_frames;
    if (s->error != MM_OK) {
      r->state = REQ_FAILED;
      r->status = s->error;
      failed++;
      continue;
    }
    const size_t cnt = (size_t)rows * (size_t)r->frames;
    if (cnt && s->rblock) {  // the caller copies its part out of the block
      r->block = s->rblock;
      r->block_src = s->rblock->data + s->L.clips[i].out_off;
      s->rblock->refs.fetch_add(1);
    } else if (cnt) {
      r->result = (float *)malloc(sizeof(float) * cnt);
      if (!r->result) {
        r->state = REQ_FAILED;
        r->status = MM_ERR_ALLOC_FAILED;
        failed++;
        continue;
      }
      memcpy(r->result, s->pinned + sizeof(float) * (size_t)s->L.clips[i].out_off, sizeof(float) * cnt);
    }
    r->state = REQ_DONE;
    r->status = MM_OK;
    completed++;
    audio_s += (double)r->length / (double)r->g.sr;
    lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
  }
  for (Request *r : s->reqs) {  // the samples are on the device (or the batch failed)
    if (r->pin) pool->put(r->pin, r->pin_cls);
    r->pin = nullptr;
    r->borrowed = nullptr;
    std::vector<float>().swap(r->signal);
  }
  if (s->rblock && s->rblock->refs.load() == 0) {  // no request took a part (or the batch failed)
    pool->put(s->rblock->data, s->rblock->cls);
    delete s->rblock;
  }
  s->rblock = nullptr;
  if (s->arena) cudaFreeAsync(s->arena, s->stream);
  s->arena = nullptr;
  in_use -= s->arena_size;
  s->arena_size = 0;
  s->reqs.clear();
  s->busy = false;
  done_cv.notify_all();
}

void Server::run() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    bool any_busy = false;
    for (Slot *s : slots) {
      if (s->busy && s->finished.load()) finish(s);
      any_busy |= s->busy;
    }
    if (stop && !any_busy) break;
    bool launched = false;
    if (!stop)
      while (admit_one(lk)) launched = true;
    if (launched) continue;
    cv.wait(lk);
  }
}

// Drops one reference to a result block; the last returns it to the pool.
void release_block(Server *srv, ResultBlock *b) {
  if (b && b->refs.fetch_sub(1) == 1) {
    srv->pool->put(b->data, b->cls);
    delete b;
  }
}

// Moves a finished request's result into *out (or returns its error) and
// deletes the request, which the caller has already taken out of srv->reqs
// (under mu); runs without the lock, so the copy out of a result block does
// not hold up the scheduler.
int32_t deliver(Server *srv, Request *r, MMBuffer *out) {
  int32_t st = r->status;
  if (r->state == REQ_DONE) {
    if (r->block) {
      const size_t cnt = (size_t)r->rows * (size_t)r->frames;
      float *data = (float *)malloc(sizeof(float) * cnt);
      if (data) {
        memcpy(data, r->block_src, sizeof(float) * cnt);
        fill_buffer(out, data, r->rows, r->frames);
      } else {
        st = MM_ERR_ALLOC_FAILED;
      }
      release_block(srv, r->block);
      r->block = nullptr;
    } else {
      fill_buffer(out, r->result, r->rows, r->frames);
      r->result = nullptr;
    }
  }
  free(r->result);
  delete r;
  return st;
}

}  // namespace

namespace {
// Queue one request: copy the samples into the pinned pool (or a pageable
// copy), or, when `borrow` is set, keep the caller's pointer.
int32_t submit_one(Server *srv, const float *signal, int64_t length, const MMFrontEndParams *params,
                   int64_t *request_id, bool borrow) {
  if (!srv || !signal || length <= 0 || !request_id) return MM_ERR_INVALID_INPUT;
  Request *r = new (std::nothrow) Request();
  if (!r) return MM_ERR_ALLOC_FAILED;
  int st = resolve_frontend(params, r->g);
  if (st == MM_OK && (r->g.n_mfcc_eff <= 0 || frame_count(length, r->g.n_fft, r->g.hop, r->g.center) == 0))
    st = MM_ERR_INVALID_INPUT;  // nothing to compute: callers use mm_mfcc for empty shapes
  if (st != MM_OK) {
    delete r;
    return st;
  }
  r->length = length;
  if (borrow) {
    r->borrowed = signal;
  } else {
    r->pin = srv->pool->get(sizeof(float) * (size_t)length, &r->pin_cls);
    if (r->pin) {
      memcpy(r->pin, signal, sizeof(float) * (size_t)length);
    } else {
      try {
        r->signal.assign(signal, signal + length);
      } catch (...) {
        delete r;
        return MM_ERR_ALLOC_FAILED;
      }
    }
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stop) {
      if (r->pin) srv->pool->put(r->pin, r->pin_cls);
      delete r;
      return MM_ERR_INVALID_INPUT;
    }
    r->id = srv->next_id++;
    srv->reqs[r->id] = r;
    srv->pending.push_back(r);
    srv->submitted++;
    *request_id = r->id;
  }
  srv->cv.notify_all();
  return MM_OK;
}
}  // namespace

extern "C" {

mm_server mm_server_create(const MMServerConfig *cfg, int32_t *status) {
  int dummy;
  int32_t *st = status ? status : &dummy;
  *st = gpu_available();
  if (*st != MM_OK) return nullptr;
  Server *srv = new (std::nothrow) Server();
  if (!srv) {
    *st = MM_ERR_ALLOC_FAILED;
    return nullptr;
  }
  const int64_t budget = (cfg && cfg->device_budget_bytes > 0) ? cfg->device_budget_bytes : (40LL << 30);
  const int inflight = (cfg && cfg->max_inflight > 0) ? std::min(cfg->max_inflight, 64) : 4;
  srv->budget = (size_t)budget;
  srv->max_batch = (cfg && cfg->max_batch_clips > 0) ? cfg->max_batch_clips : 256;
  srv->pool = new PinnedPool((cfg && cfg->host_pinned_bytes > 0) ? (size_t)cfg->host_pinned_bytes
                                                                 : (size_t(8) << 30));
  cudaGetDevice(&srv->device);
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = srv->device;
  cudaError_t e = cudaMemPoolCreate(&srv->mempool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = UINT64_MAX;  // never hand freed arenas back to the driver
    e = cudaMemPoolSetAttribute(srv->mempool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  for (int i = 0; i < inflight && e == cudaSuccess; i++) {
    Slot *s = new Slot();
    s->srv = srv;
    e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    srv->slots.push_back(s);
    if (e == cudaSuccess) {  // descriptors + results of a batch; grows if ever needed
      s->pinned_bytes = size_t(64) << 20;
      e = cudaMallocHost(&s->pinned, s->pinned_bytes);
    }
  }
  // Pinned host blocks and device arenas reserved up front: the first
  // minutes of serving then never wait on cudaMallocHost or on the device
  // pool growing (both only grow later, past these sizes).
  if (e == cudaSuccess)
    e = srv->pool->reserve(std::min<size_t>(size_t(1) << 30, srv->pool_cap()));
  if (e == cudaSuccess) {
    void *warm = nullptr;
    const size_t dev_reserve = std::min<size_t>(srv->budget, size_t(4) << 30);
    e = cudaMallocFromPoolAsync(&warm, dev_reserve, srv->mempool, srv->slots[0]->stream);
    if (e == cudaSuccess) e = cudaFreeAsync(warm, srv->slots[0]->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(srv->slots[0]->stream);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    for (Slot *s : srv->slots) {
      if (s->stream) cudaStreamDestroy(s->stream);
      if (s->pinned) cudaFreeHost(s->pinned);
      for (char *r : s->retired) cudaFreeHost(r);
      delete s;
    }
    if (srv->mempool) cudaMemPoolDestroy(srv->mempool);
    delete srv->pool;
    delete srv;
    *st = cuda_status(e);
    return nullptr;
  }
  srv->worker = std::thread([srv] { srv->run(); });
  *st = MM_OK;
  return srv;
}

void mm_server_destroy(mm_server server) {
  Server *srv = static_cast<Server *>(server);
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
    for (Request *r : srv->pending) {  // never started
      r->state = REQ_FAILED;
      r->status = MM_ERR_INVALID_INPUT;
    }
    srv->pending.clear();
  }
  srv->cv.notify_all();
  if (srv->worker.joinable()) srv->worker.join();  // in-flight batches finish first
  for (Slot *s : srv->slots) {
    if (s->stream) {
      cudaStreamSynchronize(s->stream);
      cudaStreamDestroy(s->stream);
    }
    if (s->pinned) cudaFreeHost(s->pinned);
    for (char *r : s->retired) cudaFreeHost(r);
    delete s;
  }
  for (auto &kv : srv->reqs) {
    free(kv.second->result);
    release_block(srv, kv.second->block);
    delete kv.second;
  }
  if (srv->mempool) cudaMemPoolDestroy(srv->mempool);
  delete srv->pool;
  delete srv;
}

int32_t mm_server_submit(mm_server server, const float *signal, int64_t length, const MMFrontEndParams *params,
                         int64_t *request_id) {
  return submit_one(static_cast<Server *>(server), signal, length, params, request_id, false);
}

int32_t mm_server_submit_borrowed(mm_server server, const float *signal, int64_t length,
                                  const MMFrontEndParams *params, int64_t *request_id) {
  return submit_one(static_cast<Server *>(server), signal, length, params, request_id, true);
}

int32_t mm_server_submit_borrowed_many(mm_server server, const float *const *signals, const int64_t *lengths,
                                       int32_t n, const MMFrontEndParams *params, int64_t *request_ids) {
  if (!server || n < 0 || (n > 0 && (!signals || !lengths || !params || !request_ids))) return MM_ERR_INVALID_INPUT;
  for (int32_t i = 0; i < n; i++) {
    const int32_t st =
        submit_one(static_cast<Server *>(server), signals[i], lengths[i], params + i, request_ids + i, true);
    if (st != MM_OK) {
      for (int32_t q = i; q < n; q++) request_ids[q] = -1;
      return st;
    }
  }
  return MM_OK;
}

int32_t mm_server_poll(mm_server server, int64_t request_id, MMBuffer *out) {
  Server *srv = static_cast<Server *>(server);
  if (!srv || !out) return MM_ERR_INVALID_INPUT;
  Request *r = nullptr;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(request_id);
    if (it == srv->reqs.end()) return MM_ERR_INVALID_INPUT;
    r = it->second;
    if (r->state == REQ_PENDING || r->state == REQ_RUNNING) return MM_PENDING;
    srv->reqs.erase(it);
    srv->done_cv.notify_all();  // a waiter on this id learns it is gone
  }
  return deliver(srv, r, out);
}

int32_t mm_server_wait(mm_server server, int64_t request_id, int32_t timeout_ms, MMBuffer *out) {
  Server *srv = static_cast<Server *>(server);
  if (!srv || !out) return MM_ERR_INVALID_INPUT;
  Request *r = nullptr;
  {
    std::unique_lock<std::mutex> lk(srv->mu);
    if (srv->reqs.find(request_id) == srv->reqs.end()) return MM_ERR_INVALID_INPUT;
    // looked up again on every wake-up: another caller may have taken the
    // result (and deleted the request) meanwhile
    auto ready = [&] {
      auto it = srv->reqs.find(request_id);
      if (it == srv->reqs.end()) return true;
      return it->second->state == REQ_DONE || it->second->state == REQ_FAILED;
    };
    if (timeout_ms < 0) srv->done_cv.wait(lk, ready);
    else if (!srv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return MM_PENDING;
    auto it = srv->reqs.find(request_id);
    if (it == srv->reqs.end()) return MM_ERR_INVALID_INPUT;  // taken by another caller
    r = it->second;
    srv->reqs.erase(it);
    srv->done_cv.notify_all();  // a second waiter on this id learns it is gone
  }
  return deliver(srv, r, out);
}

int32_t mm_server_stats(mm_server server, MMServerStats *out) {
  Server *srv = static_cast<Server *>(server);
  if (!srv || !out) return MM_ERR_INVALID_INPUT;
  std::vector<double> lat;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    out->submitted = srv->submitted;
    out->completed = srv->completed;
    out->failed = srv->failed;
    out->pending = (int64_t)srv->pending.size();
    int64_t busy = 0;
    for (Slot *s : srv->slots) busy += s->busy ? 1 : 0;
    out->inflight_batches = busy;
    out->batches_launched = srv->batches;
    out->bytes_in_use = (int64_t)srv->in_use;
    out->peak_bytes_in_use = (int64_t)srv->peak;
    out->audio_seconds_completed = srv->audio_s;
    out->scheduler_launch_ms = srv->launch_ms;
    out->scheduler_finish_ms = srv->finish_ms;
    lat = srv->lat_ms;
  }
  out->latency_p50_ms = out->latency_p99_ms = out->latency_mean_ms = out->latency_max_ms = 0.0;
  if (!lat.empty()) {
    std::sort(lat.begin(), lat.end());
    auto pct = [&lat](double p) {
      const size_t i = (size_t)std::min<double>((double)(lat.size() - 1), p * (double)(lat.size() - 1) + 0.5);
      return lat[i];
    };
    double sum = 0.0;
    for (double v : lat) sum += v;
    out->latency_p50_ms = pct(0.50);
    out->latency_p99_ms = pct(0.99);
    out->latency_mean_ms = sum / (double)lat.size();
    out->latency_max_ms = lat.back();
  }
  return MM_OK;
}

int32_t mm_server_reset_stats(mm_server server) {
  Server *srv = static_cast<Server *>(server);
  if (!srv) return MM_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->submitted = srv->completed = srv->failed = srv->batches = 0;
  srv->audio_s = 0.0;
  srv->launch_ms = srv->finish_ms = 0.0;
  srv->lat_ms.clear();
  srv->peak = srv->in_use;
  return MM_OK;
}

}  // extern "C"
