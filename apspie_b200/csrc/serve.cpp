// serve.cpp -- a query server over device-resident graphs with continuous
// batching.
//
// The reference answers one query per driver run (test/*/main.cu).  Here a
// server keeps graphs resident, accepts BFS / SSSP / MIS queries at any time
// (apspie_server_submit returns at once), and a worker thread turns the queue
// into batches:
//   * admission: a query's device state (its result row plus its share of the
//     traversal scratch) is charged against a byte budget; queries wait in
//     arrival order until the budget allows them in;
//   * coalescing: admitted BFS and SSSP queries are grouped by (graph, kind)
//     into jobs of up to 64 sources and run by apspie_batch_run in ONE
//     persistent launch; MIS queries run after it on the same stream;
//   * continuous batching: there are two batch slots, each with its own
//     context and stream.  While one slot's batch runs on the GPU, queries
//     that arrive are admitted into the other slot and launched right away,
//     so their work is queued behind (and its result copies overlap) the
//     running batch instead of waiting for it to return to the host.
// Each query's result row is copied back into the caller's host buffer and
// its latency (submit -> result in host memory) is recorded.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "apspie.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id;
  int type, graph, source;
  uint32_t seed;
  void *h_result;
  Clock::time_point t_submit;
  double latency_ms = 0;
  int status = APSPIE_OK;
  bool done = false;
  size_t bytes = 0;
  // placement in the slot's device / staging buffers
  size_t offset = 0;
};

struct GraphEntry {
  int m;
  int64_t nnz;
  const int *ptr, *ind, *tptr, *tind;
  const uint32_t *w;
  int symmetric;
};

struct Slot {
  apspie_ctx ctx = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  int32_t *d_out = nullptr;
  size_t d_bytes = 0;
  void *h_stage = nullptr;
  size_t h_bytes = 0;
  uint32_t *d_prio = nullptr;  // MIS priorities
  size_t prio_bytes = 0;
  std::vector<Request *> reqs;
  bool busy = false;
  int launch_status = APSPIE_OK;
};

}  // namespace

struct apspie_server {
  int device = 0;
  size_t budget = 0;
  int max_batch = 256;
  std::vector<GraphEntry> graphs;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request *> pending;
  std::unordered_map<uint64_t, Request *> reqs;
  uint64_t next_id = 1;
  size_t in_flight = 0;
  std::thread worker;
  bool stop = false;
  Slot slots[2];
  int max_pending = 1 << 20;
  // statistics
  uint64_t batches = 0, completed = 0, launched_jobs = 0;
  std::vector<double> latencies;
  std::string error;
};

namespace {

size_t request_bytes(const apspie_server *s, int type, int graph) {
  const GraphEntry &g = s->graphs[graph];
  size_t m = (size_t)g.m;
  switch (type) {
    case 0:  // BFS: result row + 1/64 of a multi-source BFS job's scratch
      return 4 * m + (32 * m + 12 * m + 256 * m) / 64 + 64;
    case 1:  // SSSP: distances, stamps and two queue rows per source
      return 16 * m + 64;
    default:  // MIS: result + priorities + two queues
      return 16 * m + 64;
  }
}

bool ensure_device(void **p, size_t *have, size_t want) {
  if (*have >= want) return true;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  size_t w = std::max<size_t>(want, 1 << 20);
  if (cudaMalloc(p, w) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  *have = w;
  return true;
}

bool ensure_host(void **p, size_t *have, size_t want) {
  if (*have >= want) return true;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *have = 0;
  size_t w = std::max<size_t>(want, 1 << 20);
  if (cudaMallocHost(p, w) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  *have = w;
  return true;
}

// Completes the requests of a finished slot: results to the callers'
// buffers, latencies, budget release.
void finish_slot(apspie_server *s, Slot &sl) {
  cudaError_t e = cudaEventSynchronize(sl.done);
  int st = sl.launch_status;
  if (st == APSPIE_OK && e != cudaSuccess) st = APSPIE_ERR_CUDA;
  auto now = Clock::now();
  std::lock_guard<std::mutex> lock(s->mu);
  for (Request *r : sl.reqs) {
    const GraphEntry &g = s->graphs[r->graph];
    if (st == APSPIE_OK && r->h_result)
      std::memcpy(r->h_result, (char *)sl.h_stage + r->offset, 4 * (size_t)g.m);
    r->status = st;
    r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
    r->done = true;
    s->in_flight -= r->bytes;
    if (st == APSPIE_OK) s->latencies.push_back(r->latency_ms);
    ++s->completed;
  }
  sl.reqs.clear();
  sl.busy = false;
  s->cv.notify_all();
}

// Builds and launches one batch on slot sl (requests already admitted).
int launch_slot(apspie_server *s, Slot &sl) {
  // layout: one m-row per request in the slot buffers
  size_t total = 0;
  for (Request *r : sl.reqs) {
    r->offset = total;
    total += 4 * (size_t)s->graphs[r->graph].m;
  }
  if (!ensure_device((void **)&sl.d_out, &sl.d_bytes, total) ||
      !ensure_host(&sl.h_stage, &sl.h_bytes, total))
    return APSPIE_ERR_OOM;
  // group BFS / SSSP by (graph, type); consecutive rows in the slot buffer
  std::map<std::pair<int, int>, std::vector<Request *>> groups;
  std::vector<Request *> mis;
  for (Request *r : sl.reqs) {
    if (r->type == 2)
      mis.push_back(r);
    else
      groups[{r->graph, r->type}].push_back(r);
  }
  std::vector<apspie_job> jobs;
  std::vector<std::vector<int>> srcs;
  std::vector<int32_t *> outs;
  // results of a job are contiguous rows: lay the grouped requests out again
  size_t off = 0;
  for (auto &kv : groups)
    for (Request *r : kv.second) {
      r->offset = off;
      off += 4 * (size_t)s->graphs[r->graph].m;
    }
  for (Request *r : mis) {
    r->offset = off;
    off += 4 * (size_t)s->graphs[r->graph].m;
  }
  srcs.reserve(groups.size());
  for (auto &kv : groups) {
    const GraphEntry &g = s->graphs[kv.first.first];
    std::vector<int> sv;
    for (Request *r : kv.second) sv.push_back(r->source);
    srcs.push_back(std::move(sv));
    apspie_job j;
    std::memset(&j, 0, sizeof(j));
    j.type = kv.first.second == 0 ? APSPIE_JOB_BFS : APSPIE_JOB_SSSP_U32;
    j.m = g.m;
    j.nnz = g.nnz;
    j.d_ptr = g.ptr;
    j.d_ind = g.ind;
    j.d_tptr = g.tptr;
    j.d_tind = g.tind;
    j.d_w = g.w;
    j.symmetric = g.symmetric;
    j.nsrc = (int)srcs.back().size();
    j.h_src = srcs.back().data();
    j.d_out = (int32_t *)((char *)sl.d_out + kv.second.front()->offset);
    j.alpha = -1;
    j.beta = -1;
    jobs.push_back(j);
  }
  int st = APSPIE_OK;
  if (!jobs.empty()) {
    // at most 64 device jobs per launch: split the job list if needed
    size_t first = 0;
    while (first < jobs.size() && st == APSPIE_OK) {
      size_t n = 0, parts = 0;
      while (first + n < jobs.size()) {
        size_t p = (jobs[first + n].nsrc + 63) / 64;
        if (parts + p > 64) break;
        parts += p;
        ++n;
      }
      if (n == 0) n = 1;  // a single job beyond 64 device jobs: reported as an error below
      st = apspie_batch_run(sl.ctx, (int)n, jobs.data() + first, 0);
      s->launched_jobs += n;
      first += n;
    }
  }
  for (Request *r : mis) {
    if (st != APSPIE_OK) break;
    const GraphEntry &g = s->graphs[r->graph];
    size_t pb = 4 * (size_t)g.m;
    if (!ensure_device((void **)&sl.d_prio, &sl.prio_bytes, pb)) {
      st = APSPIE_ERR_OOM;
      break;
    }
    // priorities via the host MT19937 into the staging row, then upload
    uint32_t *h = (uint32_t *)((char *)sl.h_stage + r->offset);
    cudaStreamSynchronize(sl.stream);  // the staging row may be in a pending copy
    apspie_mt19937_fill_host(r->seed, g.m, h);
    cudaMemcpyAsync(sl.d_prio, h, pb, cudaMemcpyHostToDevice, sl.stream);
    st = apspie_mis(sl.ctx, g.nnz, g.m, g.ptr, g.ind, sl.d_prio,
                    (int32_t *)((char *)sl.d_out + r->offset), 1.0f);
  }
  if (st == APSPIE_OK)
    if (cudaMemcpyAsync(sl.h_stage, sl.d_out, off, cudaMemcpyDeviceToHost, sl.stream) !=
        cudaSuccess)
      st = APSPIE_ERR_CUDA;
  cudaEventRecord(sl.done, sl.stream);
  return st;
}

void worker_main(apspie_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    // finish any slot whose batch completed
    for (Slot &sl : s->slots)
      if (sl.busy && cudaEventQuery(sl.done) != cudaErrorNotReady) finish_slot(s, sl);
    Slot *free_slot = nullptr;
    for (Slot &sl : s->slots)
      if (!sl.busy) free_slot = &sl;
    if (!free_slot) {
      // both batches in flight: wait for the older one
      Slot *older = &s->slots[0];
      finish_slot(s, *older);
      continue;
    }
    std::vector<Request *> batch;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      if (s->stop && s->pending.empty()) {
        bool idle = !s->slots[0].busy && !s->slots[1].busy;
        if (idle) return;
      }
      if (s->pending.empty()) {
        bool any_busy = s->slots[0].busy || s->slots[1].busy;
        s->cv.wait_for(lock, std::chrono::microseconds(any_busy ? 50 : 2000));
        continue;
      }
      // admit in arrival order while the budget allows
      while (!s->pending.empty() && (int)batch.size() < s->max_batch) {
        Request *r = s->pending.front();
        if (s->in_flight + r->bytes > s->budget && !(s->in_flight == 0 && batch.empty())) break;
        s->pending.pop_front();
        s->in_flight += r->bytes;
        batch.push_back(r);
      }
    }
    if (batch.empty()) {
      // over budget: wait for a running batch to release memory
      for (Slot &sl : s->slots)
        if (sl.busy) {
          finish_slot(s, sl);
          break;
        }
      continue;
    }
    free_slot->reqs = std::move(batch);
    free_slot->busy = true;
    free_slot->launch_status = launch_slot(s, *free_slot);
    ++s->batches;
  }
}

}  // namespace

extern "C" {

int apspie_server_create(int device, size_t state_budget_bytes, int max_batch,
                         apspie_server_t *out) {
  if (!out || state_budget_bytes == 0) return APSPIE_ERR_INVALID;
  *out = nullptr;
  auto *s = new (std::nothrow) apspie_server();
  if (!s) return APSPIE_ERR_OOM;
  s->device = device;
  s->budget = state_budget_bytes;
  s->max_batch = max_batch > 0 ? max_batch : 256;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return APSPIE_ERR_INVALID;
  }
  for (Slot &sl : s->slots) {
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
        apspie_ctx_create(device, sl.stream, &sl.ctx) != APSPIE_OK) {
      cudaGetLastError();
      delete s;
      return APSPIE_ERR_CUDA;
    }
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return APSPIE_OK;
}

int apspie_server_add_graph(apspie_server_t s, int m, int64_t nnz, const int *d_ptr,
                            const int *d_ind, const int *d_tptr, const int *d_tind,
                            const uint32_t *d_w, int symmetric, int *graph_id) {
  if (!s || m <= 0 || nnz < 0 || !d_ptr || (nnz > 0 && !d_ind) || !graph_id)
    return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  s->graphs.push_back(GraphEntry{m, nnz, d_ptr, d_ind, d_tptr, d_tind, d_w, symmetric});
  *graph_id = (int)s->graphs.size() - 1;
  return APSPIE_OK;
}

int apspie_server_submit(apspie_server_t s, int type, int graph, int source, uint32_t seed,
                         void *h_result, uint64_t *req_id) {
  if (!s || !req_id || type < 0 || type > 2) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->stop) return APSPIE_ERR_INVALID;
  if (graph < 0 || graph >= (int)s->graphs.size()) return APSPIE_ERR_INVALID;
  const GraphEntry &g = s->graphs[graph];
  if (type != 2 && (source < 0 || source >= g.m)) return APSPIE_ERR_INVALID;
  if (type == 1 && !g.w) return APSPIE_ERR_INVALID;
  if ((int)s->pending.size() >= s->max_pending) return APSPIE_ERR_BUSY;
  auto *r = new (std::nothrow) Request();
  if (!r) return APSPIE_ERR_OOM;
  r->id = s->next_id++;
  r->type = type;
  r->graph = graph;
  r->source = source;
  r->seed = seed;
  r->h_result = h_result;
  r->t_submit = Clock::now();
  r->bytes = request_bytes(s, type, graph);
  s->pending.push_back(r);
  s->reqs[r->id] = r;
  *req_id = r->id;
  s->cv.notify_all();
  return APSPIE_OK;
}

int apspie_server_poll(apspie_server_t s, uint64_t req_id, int *done, double *latency_ms) {
  if (!s || !done) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) return APSPIE_ERR_INVALID;
  *done = it->second->done ? 1 : 0;
  if (latency_ms) *latency_ms = it->second->latency_ms;
  if (it->second->done) {
    int st = it->second->status;
    delete it->second;
    s->reqs.erase(it);
    return st;
  }
  return APSPIE_OK;
}

int apspie_server_wait(apspie_server_t s, uint64_t req_id, double *latency_ms) {
  if (!s) return APSPIE_ERR_INVALID;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->reqs.find(req_id);
  if (it == s->reqs.end()) return APSPIE_ERR_INVALID;
  Request *r = it->second;
  // bounded: a query is abandoned after 600 s
  if (!s->cv.wait_for(lock, std::chrono::seconds(600), [&] { return r->done; }))
    return APSPIE_ERR_TIMEOUT;
  if (latency_ms) *latency_ms = r->latency_ms;
  int st = r->status;
  delete r;
  s->reqs.erase(it);
  return st;
}

int apspie_server_get_stats(apspie_server_t s, apspie_server_stats *out) {
  if (!s || !out) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  out->completed = s->completed;
  out->batches = s->batches;
  out->jobs = s->launched_jobs;
  out->pending = s->pending.size();
  out->in_flight_bytes = s->in_flight;
  std::vector<double> l = s->latencies;
  std::sort(l.begin(), l.end());
  auto q = [&](double p) {
    if (l.empty()) return 0.0;
    size_t i = (size_t)std::min<double>((double)l.size() - 1, p * (double)(l.size() - 1) + 0.5);
    return l[i];
  };
  out->p50_ms = q(0.50);
  out->p99_ms = q(0.99);
  out->max_ms = l.empty() ? 0.0 : l.back();
  return APSPIE_OK;
}

int apspie_server_reset_stats(apspie_server_t s) {
  if (!s) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  s->latencies.clear();
  s->completed = 0;
  s->batches = 0;
  s->launched_jobs = 0;
  return APSPIE_OK;
}

int apspie_server_destroy(apspie_server_t s) {
  if (!s) return APSPIE_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->device);
  for (Slot &sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.ctx) apspie_ctx_destroy(sl.ctx);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    cudaFree(sl.d_out);
    cudaFree(sl.d_prio);
    if (sl.h_stage) cudaFreeHost(sl.h_stage);
  }
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
  return APSPIE_OK;
}

}  // extern "C"
