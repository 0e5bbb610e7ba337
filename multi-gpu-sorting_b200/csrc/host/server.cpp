// Serving loop: sort requests of mixed sizes and key types arrive at any time
// (mgs_server_submit, any thread); a dispatcher thread batches them onto the
// GPU with continuous batching.
//
// * Device memory is reserved once, at creation, as `num_slots` resident
//   slots (keys + sort scratch), as many as the device budget admits. A batch
//   runs in one slot on that slot's own stream, so batches in different slots
//   overlap on the device (one slot's copies with another's kernels).
// * Admission by free HBM: a queued request waits until a slot is free; a
//   request larger than a slot is refused at submission (MGS_ERR_INVALID).
// * Coalescing: when a slot frees up, the oldest queued request opens a batch;
//   if it is small (<= coalesce_keys), every other queued small request of the
//   same key type joins it (FIFO order) while the slot has room, and the batch
//   is sorted by one segmented-sort launch sequence. Large requests run alone
//   through the device radix sort.
// * Latency of a request = completion (its slot's event has fired and the
//   dispatcher has seen it) minus submission, wall clock.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../kernels/engine_types.h"
#include "../kernels/launch.cuh"
#include "../kernels/radix_sort.cuh"
#include "context.h"
#include "mgs.h"

namespace mgs {
namespace {

using Clock = std::chrono::steady_clock;

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct Request {
  uint64_t id = 0;
  int dtype = 0;
  void* host = nullptr;
  size_t n = 0;
  Clock::time_point submitted, finished;
  enum State { kQueued, kRunning, kDone, kCancelled } state = kQueued;
  int status = MGS_OK;
};

struct Slot {
  char* base = nullptr;  // device: [offsets][keys][scratch]
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  uint32_t* d_status = nullptr;  // device status word of this slot
  uint32_t* h_status = nullptr;  // pinned mirror
  uint64_t* h_offsets = nullptr;  // pinned staging of segment offsets
  std::vector<std::shared_ptr<Request>> batch;
  bool busy = false;
};

class NullRecorder : public LaunchRecorder {
 public:
  void before(const char*, cudaStream_t) override { ++launches; }
  void after(const char*, cudaStream_t) override {}
  std::atomic<uint64_t> launches{0};
};

}  // namespace

struct Server {
  mgs_server_config cfg{};
  std::vector<Slot> slots;
  size_t slot_keys = 0;  // capacity in keys (of the widest type)
  std::mutex mu;
  std::condition_variable cv_work;  // new submissions
  std::condition_variable cv_done;  // completions
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Request>> requests;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread dispatcher;
  NullRecorder recorder;
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
    for (auto& s : slots) {
      if (s.stream) cudaStreamSynchronize(s.stream);
      if (s.done) cudaEventDestroy(s.done);
      if (s.stream) cudaStreamDestroy(s.stream);
      if (s.base) cudaFree(s.base);
      if (s.h_status) cudaFreeHost(s.h_status);
      if (s.h_offsets) cudaFreeHost(s.h_offsets);
    }
  }

  size_t slot_bytes_for(size_t cap_keys) const {
    const size_t max_req = cfg.max_batch_requests;
    size_t scratch = 0;
    for (int dt = 0; dt < 6; ++dt) {
      scratch = std::max(scratch, radix_sort_temp_bytes(dt, cap_keys));
      scratch = std::max(scratch, segmented_sort_temp_bytes(dt, cap_keys, max_req));
    }
    return align256((max_req + 1) * 8) + align256(cap_keys * 8) + scratch + 256;
  }

  // Issues one batch on slot `si` (called by the dispatcher without the lock).
  cudaError_t launch(Slot& s) {
    const int dtype = s.batch.front()->dtype;
    const size_t w = dtype_bytes(dtype);
    const size_t nreq = s.batch.size();
    char* d_offsets = s.base;
    char* d_keys = d_offsets + align256((cfg.max_batch_requests + 1) * 8);
    char* d_temp = d_keys + align256(slot_keys * 8);
    const size_t temp_bytes = s.bytes - size_t(d_temp - s.base);
    size_t total = 0;
    s.h_offsets[0] = 0;
    for (size_t i = 0; i < nreq; ++i) {
      total += s.batch[i]->n;
      s.h_offsets[i + 1] = total;
    }
    cudaError_t e = cudaMemsetAsync(s.d_status, 0, 4, s.stream);
    for (size_t i = 0; i < nreq && e == cudaSuccess; ++i)
      e = cudaMemcpyAsync(d_keys + s.h_offsets[i] * w, s.batch[i]->host, s.batch[i]->n * w, cudaMemcpyHostToDevice,
                          s.stream);
    if (e == cudaSuccess) {
      if (nreq == 1) {
        e = radix_sort(dtype, d_keys, total, d_temp, temp_bytes, s.stream, s.d_status, &recorder);
      } else {
        e = cudaMemcpyAsync(d_offsets, s.h_offsets, (nreq + 1) * 8, cudaMemcpyHostToDevice, s.stream);
        if (e == cudaSuccess)
          e = segmented_sort(dtype, d_keys, total, reinterpret_cast<const uint64_t*>(d_offsets), nreq, d_temp,
                             temp_bytes, s.stream, s.d_status, &recorder);
      }
    }
    for (size_t i = 0; i < nreq && e == cudaSuccess; ++i)
      e = cudaMemcpyAsync(s.batch[i]->host, d_keys + s.h_offsets[i] * w, s.batch[i]->n * w, cudaMemcpyDeviceToHost,
                          s.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.h_status, s.d_status, 4, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(s.done, s.stream);
    return e;
  }

  // Retires finished slots (lock held).
  bool retire() {
    bool any = false;
    for (auto& s : slots) {
      if (!s.busy) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      const auto now = Clock::now();
      int status = MGS_OK;
      if (q != cudaSuccess) {
        cudaGetLastError();
        status = MGS_ERR_CUDA;
      } else if (*s.h_status != 0) {
        status = (*s.h_status == kStatusBadInput) ? MGS_ERR_INVALID : MGS_ERR_TIMEOUT;
      }
      for (auto& r : s.batch) {
        r->state = Request::kDone;
        r->status = status;
        r->finished = now;
        ++completed;
        keys += r->n;
        latencies_us.push_back(std::chrono::duration<double, std::micro>(now - r->submitted).count());
      }
      last_done = now;
      s.batch.clear();
      s.busy = false;
      any = true;
    }
    return any;
  }

  // Forms a batch for a free slot from the queue (lock held); false if none.
  bool form_batch(Slot& s) {
    while (!queue.empty() && queue.front()->state == Request::kCancelled) queue.pop_front();
    if (queue.empty()) return false;
    auto head = queue.front();
    queue.pop_front();
    s.batch.assign(1, head);
    head->state = Request::kRunning;
    if (head->n <= cfg.coalesce_keys) {
      size_t total = head->n;
      for (auto it = queue.begin(); it != queue.end() && s.batch.size() < cfg.max_batch_requests;) {
        auto& r = *it;
        if (r->state == Request::kQueued && r->dtype == head->dtype && r->n <= cfg.coalesce_keys &&
            total + r->n <= slot_keys) {
          total += r->n;
          r->state = Request::kRunning;
          s.batch.push_back(r);
          it = queue.erase(it);
        } else {
          ++it;
        }
      }
    }
    s.busy = true;
    ++batches;
    return true;
  }

  void run() {
    cudaSetDevice(cfg.device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      bool progressed = retire();
      if (progressed) cv_done.notify_all();
      for (auto& s : slots) {
        if (s.busy) continue;
        if (!form_batch(s)) break;
        lk.unlock();
        const cudaError_t e = launch(s);
        lk.lock();
        if (e != cudaSuccess) {
          cudaGetLastError();
          for (auto& r : s.batch) {
            r->state = Request::kDone;
            r->status = (e == cudaErrorInvalidValue) ? MGS_ERR_INVALID : MGS_ERR_CUDA;
            r->finished = Clock::now();
          }
          s.batch.clear();
          s.busy = false;
          cv_done.notify_all();
        }
        progressed = true;
      }
      const bool busy = std::any_of(slots.begin(), slots.end(), [](const Slot& s) { return s.busy; });
      if (stop && queue.empty() && !busy) break;
      if (!progressed) {
        // Poll the slots' events while work is in flight; otherwise sleep until a submission.
        if (busy) {
          cv_work.wait_for(lk, std::chrono::microseconds(20));
        } else {
          cv_work.wait(lk, [&] { return stop || !queue.empty(); });
        }
      }
    }
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
  if (s.cfg.slot_keys == 0) s.cfg.slot_keys = size_t(1) << 26;
  if (s.cfg.num_slots <= 0) s.cfg.num_slots = 4;
  if (s.cfg.max_batch_requests == 0) s.cfg.max_batch_requests = 4096;
  if (s.cfg.coalesce_keys > s.cfg.slot_keys) s.cfg.coalesce_keys = s.cfg.slot_keys;
  s.slot_keys = s.cfg.slot_keys;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t budget = s.cfg.device_budget_bytes ? s.cfg.device_budget_bytes : free_b / 10 * 8;
  const size_t slot_bytes = s.slot_bytes_for(s.slot_keys);
  const int fit = int(std::min<size_t>(size_t(s.cfg.num_slots), budget / slot_bytes));
  if (fit < 1) {
    set_last_error("mgs_server_create: one slot of %zu keys needs %zu bytes, the device budget is %zu", s.slot_keys,
                   slot_bytes, budget);
    delete srv;
    return MGS_ERR_OOM;
  }
  s.slots.resize(fit);
  for (auto& sl : s.slots) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&sl.base), slot_bytes);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&sl.h_status), 256);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&sl.h_offsets), (s.cfg.max_batch_requests + 1) * 8);
    if (e != cudaSuccess) {
      cudaGetLastError();
      delete srv;
      set_last_error("mgs_server_create: %s", cudaGetErrorString(e));
      return MGS_ERR_OOM;
    }
    sl.bytes = slot_bytes;
    sl.d_status = reinterpret_cast<uint32_t*>(sl.base + slot_bytes - 256);
  }
  s.cfg.num_slots = fit;
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
  mgs::Server& s = server->impl;
  const size_t w = mgs::dtype_bytes(dtype);
  if (w == 0 || (n > 0 && !h_keys)) {
    set_last_error("mgs_server_submit: unknown dtype or null keys");
    return MGS_ERR_INVALID;
  }
  if (n * w > s.slot_keys * 8) {
    std::lock_guard<std::mutex> lk(s.mu);
    ++s.rejected;
    set_last_error("mgs_server_submit: %zu keys exceed a slot (%zu 8-byte keys)", n, s.slot_keys);
    return MGS_ERR_INVALID;
  }
  auto r = std::make_shared<mgs::Request>();
  r->dtype = dtype;
  r->host = h_keys;
  r->n = n;
  r->submitted = mgs::Clock::now();
  {
    std::lock_guard<std::mutex> lk(s.mu);
    if (s.stop) {
      set_last_error("mgs_server_submit: server is shutting down");
      return MGS_ERR_INVALID;
    }
    r->id = s.next_id++;
    if (!s.have_first) {
      s.have_first = true;
      s.first_submit = r->submitted;
    }
    ++s.submitted;
    s.requests[r->id] = r;
    if (n <= 1) {  // nothing to sort
      r->state = mgs::Request::kDone;
      r->finished = r->submitted;
      ++s.completed;
      s.latencies_us.push_back(0.0);
    } else {
      s.queue.push_back(r);
    }
    *request_id = r->id;
  }
  s.cv_work.notify_one();
  return MGS_OK;
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
