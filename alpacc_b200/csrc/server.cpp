// Request server on the batch path (alpacc_server_*): continuous batching.
//
// The reference's `--server` mode (backends/c/cli.c:153-161,
// backends/cuda/cli.cu:846-875) answers counted batches one input at a time.
// Here requests are submitted individually and whenever a worker is free it
// takes every queued request that fits its share of the device scratch budget
// and runs them as one batch (alpacc_gpu_parse_batch) on its own grammar
// handle and stream. With several workers, requests that arrive while one
// batch is on the GPU are admitted into the next worker's batch, so batches
// overlap on the device. Each result is identical to parsing its input alone.
#include <algorithm>
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

// Device scratch one input of n bytes may need at most (tokens, staging,
// brackets, productions, walk state, outputs), with a fixed part per input.
uint64_t scratch_estimate(uint64_t n) { return 96 * n + 16384; }

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
};

namespace {

void worker_loop(alpacc_server *s, int w) {
  alpacc_gpu_grammar *g = s->handles[w];
  void *pinned = nullptr;  // this worker's staging of the batch's inputs
  size_t pinned_cap = 0;
  std::vector<Request *> batch;
  std::vector<int64_t> offs;
  std::vector<alpacc_result> outs;
  for (;;) {
    batch.clear();
    {
      std::unique_lock<std::mutex> lock(s->mu);
      s->cv_work.wait(lock, [&] { return s->stopping || !s->queue.empty(); });
      if (s->queue.empty()) break;  // stopping
      uint64_t used = 0;
      while (!s->queue.empty() && batch.size() < s->max_batch) {
        Request *r = s->queue.front();
        const uint64_t need = scratch_estimate(r->data.size());
        if (!batch.empty() && used + need > s->budget_per_worker) break;  // admitted by memory budget
        used += need;
        batch.push_back(r);
        s->queue.pop_front();
      }
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
    const int rc = alpacc_gpu_parse_batch(g, buf, offs.data(), (uint32_t)batch.size(), outs.data());
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
  s->budget_per_worker = std::max<uint64_t>(scratch_budget / (uint64_t)workers, scratch_estimate(1));
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
  const int64_t v[4] = {s->batches, s->served, s->largest_batch, (int64_t)s->queue.size()};
  for (int i = 0; i < n && i < 4; i++) vals[i] = v[i];
  return 4;
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
