// Serving loop: sort requests of mixed sizes and key types arrive at any time
// (mgs_server_submit for host buffers, mgs_server_submit_device for buffers
// already in this GPU's memory, from any thread); a dispatcher thread batches
// them onto the GPU with continuous batching.
//
// * Device memory: one pool is reserved at creation (device_budget_bytes). A
//   batch takes exactly the bytes it needs from the pool (staging keys,
//   segment offsets, request table, sort scratch) and gives them back when it
//   retires. Admission is by free pool memory: the oldest queued request
//   starts as soon as a stream is free and the pool has room for its batch;
//   until then it, and everything behind it, waits (no overtaking, so a large
//   request is never starved by small ones). A request that could not fit even
//   in the empty pool is refused at submission.
// * Up to num_slots batches are in flight, each on its own stream, so batches
//   overlap on the device (one batch's copies with another's kernels). At most
//   one of them is large enough to fill the GPU by itself; while one runs, a
//   queued large request waits and the small requests behind it may start
//   (the large one is next as soon as the running one finishes).
// * Coalescing: a request of at most coalesce_keys keys opens a batch that
//   every other queued small request of a compatible key type joins (FIFO
//   order) while the pool has room: uint32 with int32, uint64 with int64
//   (signed keys have their top bit inverted on the way in and out, so they
//   sort as unsigned keys), float32 and float64 each on their own. A batch is
//   sorted by one segmented-sort launch sequence in a staging array. Larger
//   requests run alone: a device request is then sorted in place in the
//   caller's buffer, a host request in a staging copy.
// * Latency of a request = completion (its batch's event has fired and the
//   dispatcher has seen it) minus submission, wall clock.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../kernels/batch_copy.cuh"
#include "../kernels/engine_types.h"
#include "../kernels/launch.cuh"
#include "../kernels/radix_sort.cuh"
#include "context.h"
#include "mgs.h"

namespace mgs {
namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
// A batch of at least this many keys keeps every SM busy on its own (hundreds
// of onesweep tiles per pass): two of them at once only take SMs from each
// other, so at most one such batch is in flight; smaller batches run beside it.
constexpr size_t kLargeBatchKeys = size_t(1) << 22;

struct Request {
  uint64_t id = 0;
  int dtype = 0;
  void* keys = nullptr;  // host or device buffer, sorted in place
  bool on_device = false;
  size_t n = 0;
  Clock::time_point submitted, finished;
  enum State { kQueued, kRunning, kDone, kCancelled } state = kQueued;
  int status = MGS_OK;
};

// Key types that share a batch: the dtype the batch is sorted as, and whether
// a member's keys need their top bit inverted for it.
int batch_group(int dtype) {
  switch (dtype) {
    case MGS_I32: return MGS_U32;
    case MGS_I64: return MGS_U64;
    default: return dtype;
  }
}
bool needs_flip(int dtype) { return dtype == MGS_I32 || dtype == MGS_I64; }

// First-fit allocator over one device pool (offsets and sizes multiples of
// kAlign). Free blocks are kept sorted by offset and merged with neighbours.
class Pool {
 public:
  void reset(size_t bytes) {
    free_.clear();
    capacity_ = bytes / kAlign * kAlign;
    if (capacity_) free_[0] = capacity_;
  }
  size_t capacity() const { return capacity_; }
  size_t largest_free() const {
    size_t m = 0;
    for (const auto& f : free_) m = std::max(m, f.second);
    return m;
  }
  size_t free_bytes() const {
    size_t t = 0;
    for (const auto& f : free_) t += f.second;
    return t;
  }
  bool alloc(size_t bytes, size_t* offset) {
    bytes = align_up(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *offset = it->first;
      const size_t rest = it->second - bytes, at = it->first + bytes;
      free_.erase(it);
      if (rest) free_[at] = rest;
      return true;
    }
    return false;
  }
  void release(size_t offset, size_t bytes) {
    bytes = align_up(bytes);
    auto it = free_.emplace(offset, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<size_t, size_t> free_;
  size_t capacity_ = 0;
};

// Device bytes one batch needs, and where each part lies in its block.
struct BatchLayout {
  size_t status_off = 0, table_off = 0, offsets_off = 0, keys_off = 0, scratch_off = 0, scratch_bytes = 0,
         total = 0;
  bool staging = false;  // keys are sorted in a staging array (else in place in one device request)
};

BatchLayout batch_layout(int sort_dtype, size_t total_keys, size_t nreq, bool any_host) {
  BatchLayout L;
  const size_t w = dtype_bytes(sort_dtype);
  L.staging = nreq > 1 || any_host;
  size_t off = 0;
  L.status_off = off;
  off += kAlign;
  L.table_off = off;
  off += align_up(nreq * sizeof(BatchEntry));
  L.offsets_off = off;
  off += nreq > 1 ? align_up((nreq + 1) * 8) : 0;
  L.keys_off = off;
  off += L.staging ? align_up(total_keys * w) : 0;
  L.scratch_off = off;
  L.scratch_bytes = nreq > 1 ? segmented_sort_temp_bytes(sort_dtype, total_keys, nreq)
                             : radix_sort_temp_bytes(sort_dtype, total_keys);
  off += align_up(L.scratch_bytes);
  L.total = off;
  return L;
}

class CountingRecorder : public LaunchRecorder {
 public:
  void before(const char*, cudaStream_t) override { ++launches; }
  void after(const char*, cudaStream_t) override {}
  std::atomic<uint64_t> launches{0};
};

struct Batch {
  std::vector<std::shared_ptr<Request>> reqs;
  int sort_dtype = 0;
  size_t total = 0;
  BatchLayout layout;
  size_t pool_offset = 0;
};

struct Lane {  // one stream with at most one batch in flight
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  uint32_t* h_status = nullptr;     // pinned
  BatchEntry* h_table = nullptr;    // pinned staging of the request table
  uint64_t* h_offsets = nullptr;    // pinned staging of segment offsets
  std::unique_ptr<Batch> batch;
};

}  // namespace

struct Server {
  mgs_server_config cfg{};
  char* pool_base = nullptr;
  Pool pool;
  std::vector<Lane> lanes;
  std::mutex mu;
  std::condition_variable cv_work;  // new submissions
  std::condition_variable cv_done;  // completions
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> requests;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread dispatcher;
  CountingRecorder recorder;
  // statistics
  uint64_t submitted = 0, completed = 0, rejected = 0, cancelled = 0, batches = 0, keys = 0;
  std::vector<double> latencies_us;
  bool have_first = false;
  Clock::time_point first_submit, last_done;

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    if (dispatcher.joinable()) dispatcher.join();
    cudaSetDevice(cfg.device);
    for (auto& l : lanes) {
      if (l.stream) cudaStreamSynchronize(l.stream);
      if (l.done) cudaEventDestroy(l.done);
      if (l.stream) cudaStreamDestroy(l.stream);
      if (l.h_status) cudaFreeHost(l.h_status);
      if (l.h_table) cudaFreeHost(l.h_table);
      if (l.h_offsets) cudaFreeHost(l.h_offsets);
    }
    if (pool_base) cudaFree(pool_base);
  }

  // Bytes a request needs when it runs alone.
  size_t alone_bytes(int dtype, size_t n, bool on_device) const {
    return batch_layout(dtype, n, 1, !on_device).total;
  }

  // Issues a batch on a lane (dispatcher thread, lock not held).
  cudaError_t launch(Lane& l) {
    Batch& b = *l.batch;
    const BatchLayout& L = b.layout;
    char* base = pool_base + b.pool_offset;
    uint32_t* d_status = reinterpret_cast<uint32_t*>(base + L.status_off);
    BatchEntry* d_table = reinterpret_cast<BatchEntry*>(base + L.table_off);
    const size_t w = dtype_bytes(b.sort_dtype);
    const size_t nreq = b.reqs.size();
    char* d_keys = L.staging ? base + L.keys_off : static_cast<char*>(b.reqs[0]->keys);
    bool any_flip = false, any_device = false;
    size_t off = 0;
    l.h_offsets[0] = 0;
    for (size_t i = 0; i < nreq; ++i) {
      const Request& r = *b.reqs[i];
      l.h_table[i] = BatchEntry{r.on_device ? r.keys : nullptr, off, r.n, needs_flip(r.dtype) ? 1u : 0u, 0u};
      any_flip |= needs_flip(r.dtype) && nreq > 1;
      any_device |= r.on_device;
      off += r.n;
      l.h_offsets[i + 1] = off;
    }
    const bool staged_device = L.staging && any_device;
    const bool stage_kernels = staged_device || any_flip;
    cudaStream_t s = l.stream;
    cudaError_t e = cudaMemsetAsync(d_status, 0, 4, s);
    if (e == cudaSuccess && stage_kernels)
      e = cudaMemcpyAsync(d_table, l.h_table, nreq * sizeof(BatchEntry), cudaMemcpyHostToDevice, s);
    for (size_t i = 0; i < nreq && e == cudaSuccess; ++i) {
      const Request& r = *b.reqs[i];
      if (!r.on_device)
        e = cudaMemcpyAsync(d_keys + l.h_table[i].offset * w, r.keys, r.n * w, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess && stage_kernels) e = batch_stage_in(d_keys, d_table, uint32_t(nreq), int(w), s, &recorder);
    if (e == cudaSuccess) {
      void* scratch = base + L.scratch_off;
      if (nreq == 1) {
        // alone: the request's own key type (no transform), in place or in the staging copy
        e = radix_sort(b.reqs[0]->dtype, d_keys, b.total, scratch, L.scratch_bytes, s, d_status, &recorder);
      } else {
        char* d_offsets = base + L.offsets_off;
        e = cudaMemcpyAsync(d_offsets, l.h_offsets, (nreq + 1) * 8, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
          e = segmented_sort(b.sort_dtype, d_keys, b.total, reinterpret_cast<const uint64_t*>(d_offsets), nreq,
                             scratch, L.scratch_bytes, s, d_status, &recorder);
      }
    }
    if (e == cudaSuccess && stage_kernels) e = batch_stage_out(d_keys, d_table, uint32_t(nreq), int(w), s, &recorder);
    for (size_t i = 0; i < nreq && e == cudaSuccess; ++i) {
      const Request& r = *b.reqs[i];
      if (!r.on_device)
        e = cudaMemcpyAsync(r.keys, d_keys + l.h_table[i].offset * w, r.n * w, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(l.h_status, d_status, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(l.done, s);
    return e;
  }

  void finish(Lane& l, int status, Clock::time_point now) {
    for (auto& r : l.batch->reqs) {
      r->state = Request::kDone;
      r->status = status;
      r->finished = now;
      ++completed;
      keys += r->n;
      latencies_us.push_back(std::chrono::duration<double, std::micro>(now - r->submitted).count());
    }
    last_done = now;
    pool.release(l.batch->pool_offset, l.batch->layout.total);
    l.batch.reset();
  }

  // Retires finished batches (lock held).
  bool retire() {
    bool any = false;
    for (auto& l : lanes) {
      if (!l.batch) continue;
      const cudaError_t q = cudaEventQuery(l.done);
      if (q == cudaErrorNotReady) continue;
      int status = MGS_OK;
      if (q != cudaSuccess) {
        cudaGetLastError();
        status = MGS_ERR_CUDA;
      } else if (*l.h_status != 0) {
        status = (*l.h_status == kStatusBadInput) ? MGS_ERR_INVALID : MGS_ERR_TIMEOUT;
      }
      finish(l, status, Clock::now());
      any = true;
    }
    return any;
  }

  // Forms the next batch from the queue for a free lane (lock held): the oldest
  // request that may start (the oldest of all unless it is large while a large
  // batch runs; then the oldest small one), plus compatible small ones while
  // the pool has room. Returns null when nothing may start, or when the chosen
  // request does not fit in the pool yet.
  std::unique_ptr<Batch> form_batch() {
    while (!queue.empty() && queue.front()->state == Request::kCancelled) queue.pop_front();
    if (queue.empty()) return nullptr;
    const bool large_running = std::any_of(lanes.begin(), lanes.end(), [](const Lane& l) {
      return l.batch && l.batch->total >= kLargeBatchKeys;
    });
    std::shared_ptr<Request> head;
    for (const auto& r : queue) {
      if (r->state != Request::kQueued) continue;
      if (r->n < kLargeBatchKeys || !large_running) {
        head = r;
        break;
      }
    }
    if (!head) return nullptr;
    auto b = std::make_unique<Batch>();
    b->reqs.assign(1, head);
    b->sort_dtype = head->dtype;
    b->total = head->n;
    bool any_host = !head->on_device;
    b->layout = batch_layout(head->dtype, head->n, 1, any_host);
    const size_t room = pool.largest_free();
    if (b->layout.total > room) return nullptr;  // wait for retirements
    if (head->n <= cfg.coalesce_keys) {
      const int group = batch_group(head->dtype);
      for (auto it = queue.begin(); it != queue.end() && b->reqs.size() < cfg.max_batch_requests; ++it) {
        const auto& r = *it;
        if (r == head || r->state != Request::kQueued || batch_group(r->dtype) != group || r->n > cfg.coalesce_keys)
          continue;
        if (large_running && b->total + r->n >= kLargeBatchKeys) continue;  // stays a small batch
        const BatchLayout L = batch_layout(group, b->total + r->n, b->reqs.size() + 1, any_host || !r->on_device);
        if (L.total > room) break;
        b->reqs.push_back(r);
        b->total += r->n;
        b->sort_dtype = group;
        any_host = any_host || !r->on_device;
        b->layout = L;
      }
    }
    for (auto& r : b->reqs) r->state = Request::kRunning;
    queue.erase(std::remove_if(queue.begin(), queue.end(),
                               [](const std::shared_ptr<Request>& r) { return r->state == Request::kRunning; }),
                queue.end());
    const bool ok = pool.alloc(b->layout.total, &b->pool_offset);
    (void)ok;  // room was checked against the largest free block
    ++batches;
    return b;
  }

  void run() {
    cudaSetDevice(cfg.device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      bool progressed = retire();
      if (progressed) cv_done.notify_all();
      for (auto& l : lanes) {
        if (l.batch) continue;
        l.batch = form_batch();
        if (!l.batch) break;
        lk.unlock();
        const cudaError_t e = launch(l);
        lk.lock();
        if (e != cudaSuccess) {
          cudaGetLastError();
          cudaStreamSynchronize(l.stream);  // nothing of the batch may still run when its memory is reused
          cudaGetLastError();
          finish(l, (e == cudaErrorInvalidValue) ? MGS_ERR_INVALID : MGS_ERR_CUDA, Clock::now());
          cv_done.notify_all();
        }
        progressed = true;
      }
      const bool busy = std::any_of(lanes.begin(), lanes.end(), [](const Lane& l) { return bool(l.batch); });
      if (stop && queue.empty() && !busy) break;
      if (!progressed) {
        // Poll the batches' events while work is in flight; otherwise sleep until a submission.
        if (busy) {
          cv_work.wait_for(lk, std::chrono::microseconds(20));
        } else {
          cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        }
      }
    }
  }

  int submit(int dtype, void* keys_ptr, size_t n, bool on_device, uint64_t* request_id) {
    const size_t w = dtype_bytes(dtype);
    if (w == 0 || (n > 0 && !keys_ptr)) {
      set_last_error("mgs_server_submit: unknown dtype or null keys");
      return MGS_ERR_INVALID;
    }
    if (on_device && reinterpret_cast<uintptr_t>(keys_ptr) % w != 0) {
      set_last_error("mgs_server_submit_device: d_keys is not key-aligned");
      return MGS_ERR_INVALID;
    }
    const size_t need = n > 1 ? alone_bytes(dtype, n, on_device) : 0;
    if ((cfg.slot_keys && n > cfg.slot_keys) || n >= (size_t(1) << 32) || need > pool.capacity()) {
      std::lock_guard<std::mutex> lk(mu);
      ++rejected;
      set_last_error("mgs_server_submit: %zu keys exceed the server's limit (at most %zu keys; %zu bytes needed, the "
                     "pool holds %zu)",
                     n, cfg.slot_keys, need, pool.capacity());
      return MGS_ERR_INVALID;
    }
    auto r = std::make_shared<Request>();
    r->dtype = dtype;
    r->keys = keys_ptr;
    r->on_device = on_device;
    r->n = n;
    r->submitted = Clock::now();
    {
      std::lock_guard<std::mutex> lk(mu);
      if (stop) {
        set_last_error("mgs_server_submit: server is shutting down");
        return MGS_ERR_INVALID;
      }
      r->id = next_id++;
      if (!have_first) {
        have_first = true;
        first_submit = r->submitted;
      }
      ++submitted;
      requests[r->id] = r;
      if (n <= 1) {  // nothing to sort
        r->state = Request::kDone;
        r->finished = r->submitted;
        ++completed;
        latencies_us.push_back(0.0);
      } else {
        queue.push_back(r);
      }
      *request_id = r->id;
    }
    cv_work.notify_one();
    return MGS_OK;
  }
};

}  // namespace mgs

struct mgs_server {
  mgs::Server impl;
};

using mgs::set_last_error;

extern "C" {

int mgs_server_create(const mgs_server_config* config, mgs_server** out) {
  if (!config || !out) {
    set_last_error("mgs_server_create: null argument");
    return MGS_ERR_INVALID;
  }
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || config->device < 0 || config->device >= count) {
    cudaGetLastError();
    set_last_error("mgs_server_create: no CUDA device %d", config->device);
    return MGS_ERR_NO_DEVICE;
  }
  cudaSetDevice(config->device);
  auto* srv = new mgs_server();
  mgs::Server& s = srv->impl;
  s.cfg = *config;
  if (s.cfg.num_slots <= 0) s.cfg.num_slots = 4;
  if (s.cfg.max_batch_requests == 0) s.cfg.max_batch_requests = 4096;
  if (s.cfg.slot_keys && s.cfg.coalesce_keys > s.cfg.slot_keys) s.cfg.coalesce_keys = s.cfg.slot_keys;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  size_t budget = s.cfg.device_budget_bytes;
  if (budget == 0) budget = std::min(free_b / 2, size_t(32) << 30);
  budget = budget / mgs::kAlign * mgs::kAlign;
  cudaError_t e = budget ? cudaMalloc(reinterpret_cast<void**>(&s.pool_base), budget) : cudaErrorMemoryAllocation;
  if (e != cudaSuccess) {
    cudaGetLastError();
    s.pool_base = nullptr;
    set_last_error("mgs_server_create: cannot reserve a device pool of %zu bytes (%zu free)", budget, free_b);
    delete srv;
    return MGS_ERR_OOM;
  }
  s.pool.reset(budget);
  s.cfg.device_budget_bytes = budget;
  s.lanes.resize(size_t(s.cfg.num_slots));
  for (auto& l : s.lanes) {
    e = cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&l.h_status), 256);
    if (e == cudaSuccess)
      e = cudaMallocHost(reinterpret_cast<void**>(&l.h_table), s.cfg.max_batch_requests * sizeof(mgs::BatchEntry));
    if (e == cudaSuccess)
      e = cudaMallocHost(reinterpret_cast<void**>(&l.h_offsets), (s.cfg.max_batch_requests + 1) * 8);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_last_error("mgs_server_create: %s", cudaGetErrorString(e));
      delete srv;
      return MGS_ERR_OOM;
    }
  }
  s.dispatcher = std::thread([&s] { s.run(); });
  *out = srv;
  mgs::clear_last_error();
  return MGS_OK;
}

int mgs_server_destroy(mgs_server* server) {
  delete server;  // drains queued and running requests first
  return MGS_OK;
}

int mgs_server_submit(mgs_server* server, int dtype, void* h_keys, size_t n, uint64_t* request_id) {
  if (!server || !request_id) {
    set_last_error("mgs_server_submit: null argument");
    return MGS_ERR_INVALID;
  }
  return server->impl.submit(dtype, h_keys, n, false, request_id);
}

int mgs_server_submit_device(mgs_server* server, int dtype, void* d_keys, size_t n, uint64_t* request_id) {
  if (!server || !request_id) {
    set_last_error("mgs_server_submit_device: null argument");
    return MGS_ERR_INVALID;
  }
  return server->impl.submit(dtype, d_keys, n, true, request_id);
}

int mgs_server_wait(mgs_server* server, uint64_t request_id, int timeout_ms, int* request_status) {
  if (!server) {
    set_last_error("mgs_server_wait: server is null");
    return MGS_ERR_INVALID;
  }
  mgs::Server& s = server->impl;
  std::unique_lock<std::mutex> lk(s.mu);
  auto it = s.requests.find(request_id);
  if (it == s.requests.end()) {
    set_last_error("mgs_server_wait: unknown request %llu", static_cast<unsigned long long>(request_id));
    return MGS_ERR_INVALID;
  }
  auto r = it->second;
  auto finished = [&] { return r->state == mgs::Request::kDone || r->state == mgs::Request::kCancelled; };
  if (timeout_ms < 0) {
    s.cv_done.wait(lk, finished);
  } else if (!s.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished)) {
    set_last_error("mgs_server_wait: request %llu not finished after %d ms",
                   static_cast<unsigned long long>(request_id), timeout_ms);
    return MGS_ERR_TIMEOUT;
  }
  const int st = r->state == mgs::Request::kCancelled ? MGS_ERR_CANCELLED : r->status;
  if (request_status) *request_status = st;
  s.requests.erase(request_id);
  return MGS_OK;
}

int mgs_server_cancel(mgs_server* server, uint64_t request_id) {
  if (!server) {
    set_last_error("mgs_server_cancel: server is null");
    return MGS_ERR_INVALID;
  }
  mgs::Server& s = server->impl;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    auto it = s.requests.find(request_id);
    if (it == s.requests.end()) {
      set_last_error("mgs_server_cancel: unknown request");
      return MGS_ERR_INVALID;
    }
    if (it->second->state != mgs::Request::kQueued) {
      set_last_error("mgs_server_cancel: request already running or finished");
      return MGS_ERR_BUSY;
    }
    it->second->state = mgs::Request::kCancelled;
    ++s.cancelled;
  }
  s.cv_done.notify_all();
  return MGS_OK;
}

int mgs_server_stats_get(mgs_server* server, mgs_server_stats* out, int reset) {
  if (!server || !out) {
    set_last_error("mgs_server_stats_get: null argument");
    return MGS_ERR_INVALID;
  }
  mgs::Server& s = server->impl;
  std::lock_guard<std::mutex> lk(s.mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s.submitted;
  out->completed = s.completed;
  out->rejected = s.rejected;
  out->cancelled = s.cancelled;
  out->batches = s.batches;
  out->keys = s.keys;
  out->kernel_launches = s.recorder.launches.load();
  out->num_slots = s.cfg.num_slots;
  out->pool_bytes = s.pool.capacity();
  out->pool_free_bytes = s.pool.free_bytes();
  std::vector<double> lat = s.latencies_us;
  if (!lat.empty()) {
    auto pct = [&](double p) {
      const size_t k = std::min(lat.size() - 1, size_t(p * double(lat.size() - 1) + 0.5));
      std::nth_element(lat.begin(), lat.begin() + k, lat.end());
      return lat[k];
    };
    out->p50_us = pct(0.50);
    out->p99_us = pct(0.99);
    double sum = 0, mx = 0;
    for (double v : s.latencies_us) {
      sum += v;
      mx = std::max(mx, v);
    }
    out->mean_us = sum / double(s.latencies_us.size());
    out->max_us = mx;
  }
  if (s.have_first && s.completed > 0)
    out->busy_s = std::chrono::duration<double>(s.last_done - s.first_submit).count();
  if (reset) {
    s.submitted = s.completed = s.rejected = s.cancelled = s.batches = s.keys = 0;
    s.latencies_us.clear();
    s.have_first = false;
    s.recorder.launches = 0;
  }
  return MGS_OK;
}

}  // extern "C"
