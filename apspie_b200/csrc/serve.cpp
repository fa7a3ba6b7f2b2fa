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
// Each query's result row is copied into the caller's host buffer, or into
// its device buffer (or dropped, for load tests), and its latency (submit ->
// result in host / device memory) is recorded.  MIS priorities (mt19937 of
// the query's seed) are generated once per (graph, seed) and kept on the
// device.
//
// apspie_server_replay drives the server with a timed query stream (open
// loop: each query is submitted at its scheduled arrival time, and its
// latency counts from that time); apspie_server_replay_plain runs the same
// stream one query at a time through the single-source kernels, for
// comparison.
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
  int32_t *d_result = nullptr;
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
  // MIS priorities per (graph, seed), on the device
  std::mutex prio_mu;
  std::map<std::pair<int, uint32_t>, uint32_t *> prio_cache;
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

// Device priorities of an MIS query: mt19937(seed) for the graph's vertices,
// generated on the host and uploaded on `stream` the first time.
int get_prio(apspie_server *s, int graph, uint32_t seed, cudaStream_t stream, uint32_t **out) {
  std::lock_guard<std::mutex> lock(s->prio_mu);
  auto key = std::make_pair(graph, seed);
  auto it = s->prio_cache.find(key);
  if (it != s->prio_cache.end()) {
    *out = it->second;
    return APSPIE_OK;
  }
  const size_t m = (size_t)s->graphs[graph].m;
  uint32_t *d = nullptr, *h = nullptr;
  if (cudaMalloc(&d, 4 * m) != cudaSuccess || cudaMallocHost(&h, 4 * m) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(d);
    return APSPIE_ERR_OOM;
  }
  int st = apspie_mt19937_fill_host(seed, (int64_t)m, h);
  if (st == APSPIE_OK && (cudaMemcpyAsync(d, h, 4 * m, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
                          cudaStreamSynchronize(stream) != cudaSuccess)) {
    cudaGetLastError();
    st = APSPIE_ERR_CUDA;
  }
  cudaFreeHost(h);
  if (st != APSPIE_OK) {
    cudaFree(d);
    return st;
  }
  s->prio_cache[key] = d;
  *out = d;
  return APSPIE_OK;
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
    uint32_t *prio = nullptr;
    st = get_prio(s, r->graph, r->seed, sl.stream, &prio);
    if (st == APSPIE_OK)
      st = apspie_mis(sl.ctx, g.nnz, g.m, g.ptr, g.ind, prio,
                      (int32_t *)((char *)sl.d_out + r->offset), 1.0f);
  }
  // results to the callers: host rows through the staging buffer, device
  // rows directly; a query with neither only has its latency recorded
  for (Request *r : sl.reqs) {
    if (st != APSPIE_OK) break;
    const size_t bytes = 4 * (size_t)s->graphs[r->graph].m;
    cudaError_t e = cudaSuccess;
    if (r->h_result)
      e = cudaMemcpyAsync((char *)sl.h_stage + r->offset, (char *)sl.d_out + r->offset, bytes,
                          cudaMemcpyDeviceToHost, sl.stream);
    if (e == cudaSuccess && r->d_result)
      e = cudaMemcpyAsync(r->d_result, (char *)sl.d_out + r->offset, bytes,
                          cudaMemcpyDeviceToDevice, sl.stream);
    if (e != cudaSuccess) st = APSPIE_ERR_CUDA;
  }
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

}  // extern "C"

namespace {

int check_query(apspie_server *s, int type, int graph, int source) {
  if (type < 0 || type > 2) return APSPIE_ERR_INVALID;
  if (graph < 0 || graph >= (int)s->graphs.size()) return APSPIE_ERR_INVALID;
  const GraphEntry &g = s->graphs[graph];
  if (type != 2 && (source < 0 || source >= g.m)) return APSPIE_ERR_INVALID;
  if (type == 1 && !g.w) return APSPIE_ERR_INVALID;
  return APSPIE_OK;
}

// Queues one query (caller holds s->mu).
int enqueue_locked(apspie_server *s, int type, int graph, int source, uint32_t seed,
                   void *h_result, int32_t *d_result, Clock::time_point t_submit, Request **out) {
  if (s->stop) return APSPIE_ERR_INVALID;
  int st = check_query(s, type, graph, source);
  if (st) return st;
  if ((int)s->pending.size() >= s->max_pending) return APSPIE_ERR_BUSY;
  auto *r = new (std::nothrow) Request();
  if (!r) return APSPIE_ERR_OOM;
  r->id = s->next_id++;
  r->type = type;
  r->graph = graph;
  r->source = source;
  r->seed = seed;
  r->h_result = h_result;
  r->d_result = d_result;
  r->t_submit = t_submit;
  r->bytes = request_bytes(s, type, graph);
  s->pending.push_back(r);
  s->reqs[r->id] = r;
  *out = r;
  s->cv.notify_all();
  return APSPIE_OK;
}

void spin_until(Clock::time_point t) {
  while (Clock::now() < t) std::this_thread::yield();
}

}  // namespace

extern "C" {

int apspie_server_submit(apspie_server_t s, int type, int graph, int source, uint32_t seed,
                         void *h_result, uint64_t *req_id) {
  if (!s || !req_id) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  Request *r = nullptr;
  int st = enqueue_locked(s, type, graph, source, seed, h_result, nullptr, Clock::now(), &r);
  if (st == APSPIE_OK) *req_id = r->id;
  return st;
}

int apspie_server_submit_device(apspie_server_t s, int type, int graph, int source,
                                uint32_t seed, int32_t *d_result, uint64_t *req_id) {
  if (!s || !req_id) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  Request *r = nullptr;
  int st = enqueue_locked(s, type, graph, source, seed, nullptr, d_result, Clock::now(), &r);
  if (st == APSPIE_OK) *req_id = r->id;
  return st;
}

int apspie_server_replay(apspie_server_t s, int n, const apspie_query *q, double *lat_ms,
                         double *wall_ms) {
  if (!s || n < 0 || (n > 0 && (!q || !lat_ms))) return APSPIE_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (int i = 0; i < n; ++i)
      if (check_query(s, q[i].type, q[i].graph, q[i].source) || q[i].t_us < 0 ||
          (i > 0 && q[i].t_us < q[i - 1].t_us))
        return APSPIE_ERR_INVALID;
  }
  std::vector<Request *> rs((size_t)n, nullptr);
  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(1);
  int st = APSPIE_OK;
  for (int i = 0; i < n && st == APSPIE_OK; ++i) {
    const Clock::time_point at =
        t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(q[i].t_us));
    spin_until(at);
    std::lock_guard<std::mutex> lock(s->mu);
    // the pending queue is large; a full one is waited out, the query keeps
    // its scheduled arrival time
    while ((st = enqueue_locked(s, q[i].type, q[i].graph, q[i].source, q[i].seed, nullptr,
                                nullptr, at, &rs[i])) == APSPIE_ERR_BUSY) {
      s->mu.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(100));
      s->mu.lock();
    }
  }
  double last = 0;
  std::unique_lock<std::mutex> lock(s->mu);
  for (int i = 0; i < n; ++i) {
    Request *r = rs[i];
    if (!r) {
      lat_ms[i] = -1;
      continue;
    }
    if (!s->cv.wait_for(lock, std::chrono::seconds(600), [&] { return r->done; })) {
      st = APSPIE_ERR_TIMEOUT;
      lat_ms[i] = -1;
      continue;  // left in the table; the server frees it on destroy
    }
    if (r->status != APSPIE_OK && st == APSPIE_OK) st = r->status;
    lat_ms[i] = r->latency_ms;
    last = std::max(last, std::chrono::duration<double, std::milli>(r->t_submit - t0).count() +
                              r->latency_ms);
    s->reqs.erase(r->id);
    delete r;
  }
  if (wall_ms) *wall_ms = last;
  return st;
}

int apspie_server_replay_plain(apspie_server_t s, int n, const apspie_query *q, double *lat_ms,
                               double *wall_ms) {
  if (!s || n < 0 || (n > 0 && (!q || !lat_ms))) return APSPIE_ERR_INVALID;
  int maxm = 0;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (int i = 0; i < n; ++i)
      if (check_query(s, q[i].type, q[i].graph, q[i].source) || q[i].t_us < 0 ||
          (i > 0 && q[i].t_us < q[i - 1].t_us))
        return APSPIE_ERR_INVALID;
    for (const GraphEntry &g : s->graphs) maxm = std::max(maxm, g.m);
  }
  if (cudaSetDevice(s->device) != cudaSuccess) return APSPIE_ERR_CUDA;
  cudaStream_t stream = nullptr;
  apspie_ctx ctx = nullptr;
  int32_t *row = nullptr;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&row, 4 * (size_t)std::max(maxm, 1)) != cudaSuccess) {
    cudaGetLastError();
    if (stream) cudaStreamDestroy(stream);
    return APSPIE_ERR_OOM;
  }
  int st = apspie_ctx_create(s->device, stream, &ctx);
  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(1);
  double last = 0;
  for (int i = 0; i < n && st == APSPIE_OK; ++i) {
    const Clock::time_point at =
        t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(q[i].t_us));
    spin_until(at);  // returns at once when the previous query ran late
    const GraphEntry &g = s->graphs[q[i].graph];
    if (q[i].type == 0) {
      const int *tp = g.symmetric ? g.ptr : g.tptr, *ti = g.symmetric ? g.ind : g.tind;
      st = apspie_bfs(ctx, q[i].source, g.nnz, g.m, g.ptr, g.ind, tp, ti, row, 0);
    } else if (q[i].type == 1) {
      st = apspie_sssp_u32(ctx, q[i].source, g.nnz, g.m, g.ptr, g.ind, g.w, (uint32_t *)row, 0);
    } else {
      uint32_t *prio = nullptr;
      st = get_prio(s, q[i].graph, q[i].seed, stream, &prio);
      if (st == APSPIE_OK) st = apspie_mis(ctx, g.nnz, g.m, g.ptr, g.ind, prio, row, 1.0f);
    }
    if (st == APSPIE_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = APSPIE_ERR_CUDA;
    const double l = std::chrono::duration<double, std::milli>(Clock::now() - at).count();
    lat_ms[i] = l;
    last = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
  if (ctx) apspie_ctx_destroy(ctx);
  cudaFree(row);
  cudaStreamDestroy(stream);
  if (wall_ms) *wall_ms = last;
  return st;
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
    if (sl.h_stage) cudaFreeHost(sl.h_stage);
  }
  for (auto &kv : s->prio_cache) cudaFree(kv.second);
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
  return APSPIE_OK;
}

}  // extern "C"
