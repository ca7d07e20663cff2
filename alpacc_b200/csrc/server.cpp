// Request server on the batch path (alpacc_server_*): continuous batching.
//
// The reference's `--server` mode (backends/c/cli.c:153-161,
// backends/cuda/cli.cu:846-875) answers counted batches one input at a time.
// Here requests are submitted individually and whenever a worker is free it
// takes every queued request whose batch still fits its share of the device
// scratch budget - the exact bytes the batch path grows the worker's handle
// to, so the handle never holds more than that share unless a single request
// needs more on its own - and runs them as one batch (alpacc_gpu_parse_batch) on its own grammar
// handle and stream. With several workers, requests that arrive while one
// batch is on the GPU are admitted into the next worker's batch, so batches
// overlap on the device. Each result is identical to parsing its input alone.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/alpacc_b200.h"
#include "scratch.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  std::vector<uint8_t> data;
  Clock::time_point submitted, done_at;
  int status = 0;
  bool done = false;
  bool claimed = false;  // a caller is waiting for it (only one may)
  alpacc_result res{};
};

}  // namespace

struct alpacc_server {
  std::vector<alpacc_gpu_grammar *> handles;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::unordered_map<uint64_t, Request *> reqs;
  uint64_t next_id = 1;
  uint64_t budget_per_worker = 0;
  uint32_t max_batch = 8192;
  bool stopping = false;
  int64_t batches = 0, served = 0, largest_batch = 0;
  uint64_t max_held = 0;  // most batch scratch any worker's handle held
};

namespace {

void worker_loop(alpacc_server *s, int w) {
  alpacc_gpu_grammar *g = s->handles[w];
  void *pinned = nullptr;  // this worker's staging of the batch's inputs
  size_t pinned_cap = 0;
  std::vector<Request *> batch;
  std::vector<int64_t> offs;
  std::vector<alpacc_result> outs;
  alpacc::BatchSizes sizes;
  for (;;) {
    batch.clear();
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv_work.wait(lock, [&] { return s->stopping || !s->queue.empty(); });
      if (s->queue.empty()) break;  // stopping
      alpacc::BatchSizes z;
      while (!s->queue.empty() && batch.size() < s->max_batch) {
        Request *r = s->queue.front();
        alpacc::BatchSizes z2 = z;
        z2.add(g, r->data.size());
        if (!batch.empty() && alpacc::batch_scratch_bytes(g, z2) > s->budget_per_worker) break;
        z = z2;
        batch.push_back(r);
        s->queue.pop_front();
      }
      sizes = z;
      s->batches++;
      if ((int64_t)batch.size() > s->largest_batch) s->largest_batch = (int64_t)batch.size();
    }
    offs.assign(batch.size() + 1, 0);
    for (size_t i = 0; i < batch.size(); i++) offs[i + 1] = offs[i] + (int64_t)batch[i]->data.size();
    const size_t total = (size_t)offs.back();
    if (total > pinned_cap) {
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      pinned_cap = 0;
      if (cudaMallocHost(&pinned, total + total / 4 + 1) == cudaSuccess) pinned_cap = total + total / 4 + 1;
      else cudaGetLastError();
    }
    std::vector<uint8_t> fallback;
    uint8_t *buf = (uint8_t *)pinned;
    if (!pinned_cap) {  // no pinned memory: pageable staging
      fallback.resize(total + 1);
      buf = fallback.data();
    }
    for (size_t i = 0; i < batch.size(); i++)
      if (!batch[i]->data.empty()) std::memcpy(buf + offs[i], batch[i]->data.data(), batch[i]->data.size());
    outs.assign(batch.size(), alpacc_result{});
    alpacc::fit_batch_scratch(g, sizes, s->budget_per_worker);
    const int rc = alpacc_gpu_parse_batch(g, buf, offs.data(), (uint32_t)batch.size(), outs.data());
    const uint64_t held = alpacc::batch_scratch_held(g);
    const Clock::time_point now = Clock::now();
    {
      std::lock_guard<std::mutex> lock(s->mu);
      for (size_t i = 0; i < batch.size(); i++) {
        Request *r = batch[i];
        r->status = rc < 0 ? rc : (outs[i].valid ? ALPACC_OK : ALPACC_REJECT);
        r->res = outs[i];
        r->done_at = now;
        r->done = true;
        r->data.clear();
        r->data.shrink_to_fit();
      }
      s->served += (int64_t)batch.size();
      if (held > s->max_held) s->max_held = held;
    }
    s->cv_done.notify_all();
  }
  if (pinned) cudaFreeHost(pinned);
}

}  // namespace

extern "C" {

alpacc_server *alpacc_server_start(const alpacc_tables *tables, int device, int workers, uint64_t scratch_budget,
                                   int *err) {
  int dummy;
  if (!err) err = &dummy;
  if (!tables || workers < 1 || workers > 16 || tables->parts != ALPACC_PARTS_BOTH) {
    *err = ALPACC_E_INVALID;
    return nullptr;
  }
  alpacc_server *s = new alpacc_server();
  s->budget_per_worker = scratch_budget / (uint64_t)workers;
  for (int i = 0; i < workers; i++) {
    alpacc_gpu_grammar *g = alpacc_gpu_load(tables, device, 0, err);
    if (!g) {
      for (alpacc_gpu_grammar *h : s->handles) alpacc_gpu_free(h);
      delete s;
      return nullptr;
    }
    s->handles.push_back(g);
  }
  for (int i = 0; i < workers; i++) s->workers.emplace_back(worker_loop, s, i);
  *err = ALPACC_OK;
  return s;
}

int alpacc_server_submit(alpacc_server *s, const uint8_t *in, uint64_t n, uint64_t *id) {
  if (!s || !id || (n > 0 && !in) || n > (1ull << 31) - 1) return ALPACC_E_INVALID;
  Request *r = new Request();
  r->data.assign(in, in + n);
  r->submitted = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) {
      delete r;
      return ALPACC_E_INVALID;
    }
    r->id = s->next_id++;
    s->reqs[r->id] = r;
    s->queue.push_back(r);
    *id = r->id;
  }
  s->cv_work.notify_one();
  return ALPACC_OK;
}

int alpacc_server_wait(alpacc_server *s, uint64_t id, alpacc_result *out, double *latency_ms) {
  if (!s || !out) return ALPACC_E_INVALID;
  Request *r = nullptr;
  {
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || it->second->claimed) return ALPACC_E_INVALID;  // unknown, or another caller waits
    r = it->second;
    r->claimed = true;
    s->cv_done.wait(lock, [&] { return r->done; });
    s->reqs.erase(id);
  }
  *out = r->res;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->done_at - r->submitted).count();
  const int status = r->status;
  delete r;
  return status;
}

int alpacc_server_stats(alpacc_server *s, int64_t *vals, int n) {
  if (!s || !vals) return ALPACC_E_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  const int64_t v[6] = {s->batches,        s->served,           s->largest_batch, (int64_t)s->queue.size(),
                        (int64_t)s->max_held, (int64_t)s->budget_per_worker};
  for (int i = 0; i < n && i < 6; i++) vals[i] = v[i];
  return 6;
}

void alpacc_server_stop(alpacc_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (std::thread &t : s->workers) t.join();
  for (auto &kv : s->reqs) {  // requests nobody waited for
    alpacc_result_free(&kv.second->res);
    delete kv.second;
  }
  for (alpacc_gpu_grammar *g : s->handles) alpacc_gpu_free(g);
  delete s;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Trace replay (load generation for measurement)
// ---------------------------------------------------------------------------

namespace {

// Sleeps until t, spinning for the last 100 microseconds (sleep_until alone
// wakes tens of microseconds late, more than the gap between arrivals at high
// rates).
void wait_until(Clock::time_point t) {
  for (;;) {
    const Clock::time_point now = Clock::now();
    if (now >= t) return;
    if (t - now > std::chrono::microseconds(200)) std::this_thread::sleep_for(t - now - std::chrono::microseconds(100));
  }
}

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

extern "C" {

int alpacc_server_replay(alpacc_server *s, const uint8_t *bytes, const int64_t *offsets, const uint32_t *doc,
                         uint64_t count, const double *arrival_s, double *latency_ms, int *status,
                         double *elapsed_s) {
  if (!s || !offsets || !doc || !arrival_s || !latency_ms || !status) return ALPACC_E_INVALID;
  std::vector<uint64_t> ids(count, 0);
  std::vector<Clock::time_point> sub_at(count);
  std::atomic<uint64_t> submitted{0};
  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(2);
  auto at = [&](uint64_t i) { return t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i])); };
  std::thread sub([&] {
    for (uint64_t i = 0; i < count; i++) {
      wait_until(at(i));
      const uint32_t d = doc[i];
      const uint64_t n = (uint64_t)(offsets[d + 1] - offsets[d]);
      sub_at[i] = Clock::now();
      if (alpacc_server_submit(s, n ? bytes + offsets[d] : nullptr, n, &ids[i]) != ALPACC_OK) ids[i] = 0;
      submitted.store(i + 1, std::memory_order_release);
    }
  });
  Clock::time_point last = t0;
  for (uint64_t i = 0; i < count; i++) {
    while (submitted.load(std::memory_order_acquire) <= i) std::this_thread::yield();
    if (!ids[i]) {
      status[i] = ALPACC_E_INVALID;
      latency_ms[i] = -1.0;
      continue;
    }
    alpacc_result r{};
    double ms = 0;
    status[i] = alpacc_server_wait(s, ids[i], &r, &ms);
    alpacc_result_free(&r);
    // from the scheduled arrival: the time the submitter lagged counts
    const Clock::time_point done = sub_at[i] + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::milli>(ms));
    latency_ms[i] = ms_between(at(i), done);
    if (done > last) last = done;
  }
  sub.join();
  if (elapsed_s) *elapsed_s = std::chrono::duration<double>(last - t0).count();
  return ALPACC_OK;
}

int alpacc_gpu_replay(alpacc_gpu_grammar *g, const uint8_t *bytes, const int64_t *offsets, const uint32_t *doc,
                      uint64_t count, const double *arrival_s, double *latency_ms, int *status, double *elapsed_s) {
  if (!g || !offsets || !doc || !arrival_s || !latency_ms || !status) return ALPACC_E_INVALID;
  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(2);
  Clock::time_point last = t0;
  for (uint64_t i = 0; i < count; i++) {
    const Clock::time_point at =
        t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
    wait_until(at);
    const uint32_t d = doc[i];
    const uint64_t n = (uint64_t)(offsets[d + 1] - offsets[d]);
    alpacc_result r{};
    status[i] = alpacc_gpu_parse(g, n ? bytes + offsets[d] : nullptr, n, &r);
    alpacc_result_free(&r);
    last = Clock::now();
    latency_ms[i] = ms_between(at, last);
  }
  if (elapsed_s) *elapsed_s = std::chrono::duration<double>(last - t0).count();
  return ALPACC_OK;
}

}  // extern "C"
