// serve.cpp -- a query server over device-resident graphs with continuous
// batching.
//
// The reference answers one query per driver run (test/*/main.cu).  Here a
// server keeps graphs resident, accepts BFS / SSSP / MIS queries at any time
// (apspie_server_submit returns at once), and a worker thread turns the queue
// into batches:
//   * admission: a query's device state (its result row plus its share of the
//     traversal scratch) is charged against a byte budget and against the
//     device memory the server can use: what its lanes already hold plus the
//     device's free memory (cudaMemGetInfo, read when a batch forms, at most
//     every 10 ms), less a 2 GiB reserve; queries wait in arrival
//     order until both allow them in;
//   * coalescing: the admitted BFS and SSSP queries of one (graph, kind) form
//     a group, run by ONE apspie_batch_run (multi-source frontier matrix), or
//     by the single-source kernel when the group has one query (or, on the
//     largest graphs, fewer than the group size from which the batch pays);
//     the MIS queries of one (graph, seed) are one computation whose
//     membership row is copied to each of them.  Groups are launched cheapest first
//     (measured time per group, kept per graph and kind), and each group has
//     its own completion event, so a quick query is not held back by a slow
//     one of the same batch;
//   * lanes: graphs whose traversals take many levels (found when the graph
//     is added, by one probe BFS) run on a second stream with a quarter of
//     the GPU's persistent blocks, next to the main lane with the rest, so
//     their thousands of short levels do not keep the whole GPU from the
//     other queries; while no such traversal is in the batch or running in
//     the other slot, the main lane takes the whole GPU;
//   * continuous batching: there are two batch slots.  While one slot's
//     groups run, queries that arrive are admitted into the other slot,
//     which is launched, queued on the GPU behind (and overlapping the
//     copies of) the running groups, once the running slot's main lane is
//     down to its last group; until then the queries keep gathering, so
//     under load the groups grow instead of the batches multiplying.
// The worker never blocks on one group: between rounds it pauses briefly
// and polls every running group's completion event, so a finished query is
// reported within tens of microseconds whichever slot it ran in.
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
#include <new>
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
  bool to_stage = false;  // result copied to the slot's pinned staging rows only (replay)
  Clock::time_point t_submit;
  double latency_ms = 0;
  int status = APSPIE_OK;
  bool done = false;
  size_t bytes = 0;
  size_t dev_off = 0;   // result row in the slot's device buffer
  size_t host_off = 0;  // ... and in its pinned staging buffer (host results)
};

// A graph traversal is "deep" when a probe BFS takes more levels than this:
// its queries go to the small-grid lane.
constexpr int kDeepLevels = 64;

struct GraphEntry {
  int m;
  int64_t nnz;
  const int *ptr, *ind, *tptr, *tind;
  const uint32_t *w;
  int symmetric;
  bool deep;
  float cost_ms[3];  // running estimate of one group's device time, per kind
  // in-adjacency with its weights for push/pull SSSP (apspie_server_set_sssp_in)
  const int *stptr = nullptr, *stind = nullptr;
  const uint32_t *stw = nullptr;
};

// On graphs with more edges than kLargeNnz, BFS and SSSP groups smaller
// than these run their queries one by one through the single-source
// kernels: the multi-source launch shares little there (measured, time per
// query against one by one: R-MAT 23 BFS 0.72x at 8 sources, 1.29x at 16,
// 2.9x at 64; SSSP 0.93 - 0.98x at 4 - 8, 1.16x at 16, 1.24x at 32; R-MAT 22
// BFS 1.5x from 8 sources, SSSP 1.09x at 8 - 16), while on smaller graphs
// the batch wins from two queries on.
constexpr int64_t kLargeNnz = 64ll << 20;
constexpr size_t kBfsBatchMinGroup = 12;
constexpr size_t kSsspBatchMinGroup = 16;

// One SSSP query through the single-source kernel, push/pull when the
// graph's in-adjacency with weights was registered.
int sssp_one(apspie_ctx ctx, const GraphEntry &ge, int src, uint32_t *out) {
  if (ge.stptr)
    return apspie_sssp_u32_pull(ctx, src, ge.nnz, ge.m, ge.ptr, ge.ind, ge.w, ge.stptr, ge.stind,
                                ge.stw, out, 0);
  return apspie_sssp_u32(ctx, src, ge.nnz, ge.m, ge.ptr, ge.ind, ge.w, out, 0);
}

struct Group {
  int kind = 0, graph = 0, lane = 0;
  std::vector<Request *> reqs;
  cudaEvent_t start = nullptr, end = nullptr;
  cudaEvent_t computed = nullptr;  // the traversal's end, which the copies wait for
  int status = APSPIE_OK;
  bool done = false;
};

struct Lane {
  apspie_ctx ctx = nullptr;
  cudaStream_t stream = nullptr;
  // result copies: on a stream of their own behind each group's traversal,
  // so the copy engines move a group's rows while the next group computes
  cudaStream_t copy = nullptr;
};

struct Slot {
  Lane lane[2];
  int32_t *d_out = nullptr;
  size_t d_bytes = 0;
  void *h_stage = nullptr;
  size_t h_bytes = 0;
  std::vector<Group> groups;
  std::vector<cudaEvent_t> events;  // pool, three per group
  // set and cleared by the worker; read by warm_lanes on the thread adding a graph
  std::atomic<bool> busy{false};
};

}  // namespace

struct apspie_server {
  int device = 0;
  size_t budget = 0;
  int max_batch = 256;
  // appended by add_graph while the worker runs: read and written under mu
  std::deque<GraphEntry> graphs;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request *> pending;
  std::unordered_map<uint64_t, Request *> reqs;
  uint64_t next_id = 1;
  size_t in_flight = 0;
  std::thread worker;
  bool stop = false;
  Slot slots[2];
  bool any_deep = false;
  bool warming = false;  // add_graph is warming the lanes: the worker launches nothing
  // admission also against device memory: the query state the server may
  // hold is at most what its lanes already hold (workspaces and result
  // buffers, which admitted queries reuse) plus what is free on the device,
  // less a reserve; re-read when a batch forms, at most every 10 ms
  size_t mem_cap = 0;
  bool free_known = false;
  Clock::time_point mem_read_at{};
  int fail_next_kind = -1;  // test hook: the next group of this kind fails
  int max_pending = 1 << 20;
  // MIS priorities per (graph, seed), on the device
  std::mutex prio_mu;
  std::map<std::pair<int, uint32_t>, uint32_t *> prio_cache;
  // the plain one-query-at-a-time path of apspie_server_replay_plain: its
  // own stream, context and result rows, kept across calls so a warm-up
  // replay leaves them warm, as the server's lanes are
  cudaStream_t plain_stream = nullptr;
  apspie_ctx plain_ctx = nullptr;
  int32_t *plain_row = nullptr;
  void *plain_hrow = nullptr;
  size_t plain_m = 0;
  // statistics
  uint64_t batches = 0, completed = 0, launched_jobs = 0, mem_waits = 0;
  double max_launch_ms = 0.0;  // longest host time of one launch_slot
  // outgrown result and staging buffers (device, pinned host), freed at destroy
  std::vector<void *> retired, retired_host;
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

// Grows a slot's device result buffer (host = false) or its pinned staging
// buffer (host = true).  The old buffer is kept (released when the server is
// destroyed) instead of freed: cudaFree and cudaFreeHost wait for all the
// device's work, the other slot's traversals included (a 335 ms launch was
// measured at 1,000 q/s).  Growth is at least twofold, so what is kept is
// at most the size of the current buffer.
bool ensure_buffer(void **p, size_t *have, size_t want, bool host, std::vector<void *> *retired) {
  if (*have >= want) return true;
  const size_t prev = *have;
  if (*p) retired->push_back(*p);
  *p = nullptr;
  *have = 0;
  size_t w = std::max<size_t>({want, 2 * prev, (size_t)1 << 20});
  if ((host ? cudaMallocHost(p, w) : cudaMalloc(p, w)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return false;
  }
  *have = w;
  return true;
}

// Device priorities of an MIS query: mt19937(seed) for the graph's m
// vertices, generated on the host and uploaded on `stream` the first time.
int get_prio(apspie_server *s, int graph, size_t m, uint32_t seed, cudaStream_t stream,
             uint32_t **out) {
  std::lock_guard<std::mutex> lock(s->prio_mu);
  auto key = std::make_pair(graph, seed);
  auto it = s->prio_cache.find(key);
  if (it != s->prio_cache.end()) {
    *out = it->second;
    return APSPIE_OK;
  }
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

// Levels of one BFS of graph g from its first vertex with edges, on a
// context and stream of its own (the depth of the graph's traversals).
int probe_levels(int device, const GraphEntry &g, int *levels) {
  *levels = 0;
  if (g.nnz == 0) return APSPIE_OK;
  if (cudaSetDevice(device) != cudaSuccess) return APSPIE_ERR_CUDA;
  const int nh = std::min(g.m, 4096);
  std::vector<int> h(nh + 1);
  if (cudaMemcpy(h.data(), g.ptr, sizeof(int) * (nh + 1), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return APSPIE_ERR_CUDA;
  }
  int src = -1;
  for (int u = 0; u < nh && src < 0; ++u)
    if (h[u + 1] > h[u]) src = u;
  if (src < 0) return APSPIE_OK;  // a sparse prefix: treat as shallow
  cudaStream_t stream = nullptr;
  apspie_ctx ctx = nullptr;
  int32_t *depth = nullptr;
  int st = APSPIE_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess &&
      cudaMalloc(&depth, 4 * (size_t)g.m) == cudaSuccess &&
      apspie_ctx_create(device, stream, &ctx) == APSPIE_OK) {
    const int *tp = g.tptr ? g.tptr : (g.symmetric ? g.ptr : nullptr);
    const int *ti = g.tptr ? g.tind : (g.symmetric ? g.ind : nullptr);
    st = apspie_bfs(ctx, src, g.nnz, g.m, g.ptr, g.ind, tp, ti, depth, 0);
    apspie_bfs_stats bs;
    if (st == APSPIE_OK) st = apspie_bfs_get_stats(ctx, &bs);
    if (st == APSPIE_OK) *levels = bs.levels;
  }
  cudaGetLastError();
  if (ctx) apspie_ctx_destroy(ctx);
  cudaFree(depth);
  if (stream) cudaStreamDestroy(stream);
  return st;
}

// Free device memory kept out of admission for the library's workspaces,
// result rows and staging (they grow after admission).
constexpr size_t kFreeReserve = size_t(2) << 30;

// Reads the device's free memory and the server's own holdings (worker
// thread, caller holds s->mu): queries may fill what the server holds
// plus what is free, less the reserve.  At most once per kMemReadPeriod:
// the reading is a driver call, and the cap moves only when the server or
// another user of the device allocates.
constexpr auto kMemReadPeriod = std::chrono::milliseconds(10);

void refresh_free_locked(apspie_server *s) {
  const auto now = Clock::now();
  if (s->free_known && now - s->mem_read_at < kMemReadPeriod) return;
  s->mem_read_at = now;
  size_t fr = 0, total = 0;
  if (cudaMemGetInfo(&fr, &total) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  size_t held = 0;
  for (Slot &sl : s->slots) {
    held += sl.d_bytes;
    for (Lane &ln : sl.lane) {
      size_t b = 0;
      if (ln.ctx && apspie_ctx_workspace_bytes(ln.ctx, &b) == APSPIE_OK) held += b;
    }
  }
  s->mem_cap = held + fr > kFreeReserve ? held + fr - kFreeReserve : 0;
  s->free_known = true;
}

// Completes the requests of a finished group: results to the callers'
// buffers, latencies, budget release, the group's cost estimate.
void finish_group(apspie_server *s, Slot &sl, Group &g) {
  int st = g.status;
  float ms = 0;
  if (st == APSPIE_OK && cudaEventElapsedTime(&ms, g.start, g.end) != cudaSuccess) {
    cudaGetLastError();
    st = APSPIE_ERR_CUDA;
  }
  auto now = Clock::now();
  std::lock_guard<std::mutex> lock(s->mu);
  GraphEntry &ge = s->graphs[g.graph];
  if (st == APSPIE_OK) ge.cost_ms[g.kind] = 0.5f * ge.cost_ms[g.kind] + 0.5f * ms;
  for (Request *r : g.reqs) {
    if (st == APSPIE_OK && r->h_result)
      std::memcpy(r->h_result, (char *)sl.h_stage + r->host_off, 4 * (size_t)ge.m);
    r->status = st;
    r->latency_ms = std::chrono::duration<double, std::milli>(now - r->t_submit).count();
    r->done = true;
    s->in_flight -= r->bytes;
    if (st == APSPIE_OK) s->latencies.push_back(r->latency_ms);
    ++s->completed;
  }
  g.done = true;
  s->cv.notify_all();
}

// Completes every group of the slot whose work has finished (all of them,
// waiting, when `wait`); frees the slot when none is left.
void poll_slot(apspie_server *s, Slot &sl, bool wait) {
  bool all = true;
  for (Group &g : sl.groups) {
    if (g.done) continue;
    cudaError_t e = wait ? cudaEventSynchronize(g.end) : cudaEventQuery(g.end);
    if (e == cudaErrorNotReady) {
      all = false;
      continue;
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (g.status == APSPIE_OK) g.status = APSPIE_ERR_CUDA;
    }
    finish_group(s, sl, g);
  }
  if (all) {
    sl.groups.clear();
    sl.busy = false;
  }
}

// Launches one group on its lane: the traversal into the group's rows of the
// slot buffer, then the copies to the callers, between two timing events.
int launch_group(apspie_server *s, Slot &sl, Group &g) {
  // a copy of the graph's entry: another thread may add a graph (growing the
  // table) or register its in-adjacency while the group launches
  GraphEntry ge;
  bool inject = false;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    ge = s->graphs[g.graph];
    if (s->fail_next_kind == g.kind) {
      s->fail_next_kind = -1;
      inject = true;
    }
  }
  Lane &ln = sl.lane[g.lane];
  cudaEventRecord(g.start, ln.stream);
  int st = APSPIE_OK;
  const size_t row = 4 * (size_t)ge.m;
  if (inject) {
    st = APSPIE_ERR_CUDA;  // test hook: the group fails without running
  } else if (g.kind == 2) {
    // identical queries (same graph and seed): computed once
    Request *r = g.reqs.front();
    uint32_t *prio = nullptr;
    st = get_prio(s, g.graph, (size_t)ge.m, r->seed, ln.stream, &prio);
    if (st == APSPIE_OK)
      st = apspie_mis(ln.ctx, ge.nnz, ge.m, ge.ptr, ge.ind, prio,
                      (int32_t *)((char *)sl.d_out + r->dev_off), 1.0f);
    for (size_t i = 1; i < g.reqs.size() && st == APSPIE_OK; ++i)
      if (cudaMemcpyAsync((char *)sl.d_out + g.reqs[i]->dev_off, (char *)sl.d_out + r->dev_off,
                          row, cudaMemcpyDeviceToDevice, ln.stream) != cudaSuccess)
        st = APSPIE_ERR_CUDA;
  } else if (g.reqs.size() == 1) {
    // one source: the single-source kernels are the faster path
    Request *r = g.reqs.front();
    int32_t *out = (int32_t *)((char *)sl.d_out + r->dev_off);
    if (g.kind == 0) {
      const int *tp = ge.tptr ? ge.tptr : (ge.symmetric ? ge.ptr : nullptr);
      const int *ti = ge.tptr ? ge.tind : (ge.symmetric ? ge.ind : nullptr);
      st = apspie_bfs(ln.ctx, r->source, ge.nnz, ge.m, ge.ptr, ge.ind, tp, ti, out, 0);
    } else {
      st = sssp_one(ln.ctx, ge, r->source, (uint32_t *)out);
    }
  } else if (ge.nnz > kLargeNnz &&
             g.reqs.size() < (g.kind == 1 ? kSsspBatchMinGroup : kBfsBatchMinGroup)) {
    const int *tp = ge.tptr ? ge.tptr : (ge.symmetric ? ge.ptr : nullptr);
    const int *ti = ge.tptr ? ge.tind : (ge.symmetric ? ge.ind : nullptr);
    for (Request *r : g.reqs) {
      int32_t *out = (int32_t *)((char *)sl.d_out + r->dev_off);
      st = g.kind == 1 ? sssp_one(ln.ctx, ge, r->source, (uint32_t *)out)
                       : apspie_bfs(ln.ctx, r->source, ge.nnz, ge.m, ge.ptr, ge.ind, tp, ti, out, 0);
      if (st != APSPIE_OK) break;
    }
  } else {
    std::vector<int> src;
    for (Request *r : g.reqs) src.push_back(r->source);
    apspie_job j;
    std::memset(&j, 0, sizeof(j));
    j.type = g.kind == 0 ? APSPIE_JOB_BFS : APSPIE_JOB_SSSP_U32;
    j.m = ge.m;
    j.nnz = ge.nnz;
    j.d_ptr = ge.ptr;
    j.d_ind = ge.ind;
    j.d_tptr = ge.tptr;
    j.d_tind = ge.tind;
    j.d_w = ge.w;
    j.symmetric = ge.symmetric;
    j.nsrc = (int)src.size();
    j.h_src = src.data();
    j.d_out = (int32_t *)((char *)sl.d_out + g.reqs.front()->dev_off);
    j.alpha = -1;
    j.beta = -1;
    j.d_stptr = ge.stptr;
    j.d_stind = ge.stind;
    j.d_stw = ge.stw;
    st = apspie_batch_run(ln.ctx, 1, &j, 0);
    std::lock_guard<std::mutex> lock(s->mu);
    ++s->launched_jobs;
  }
  // results to the callers, on the lane's copy stream once the traversal
  // is done: host rows through the staging buffer, device rows directly; a
  // query with neither only has its latency recorded
  cudaEventRecord(g.computed, ln.stream);
  cudaStreamWaitEvent(ln.copy, g.computed, 0);
  for (Request *r : g.reqs) {
    if (st != APSPIE_OK) break;
    cudaError_t e = cudaSuccess;
    if (r->h_result || r->to_stage)
      e = cudaMemcpyAsync((char *)sl.h_stage + r->host_off, (char *)sl.d_out + r->dev_off, row,
                          cudaMemcpyDeviceToHost, ln.copy);
    if (e == cudaSuccess && r->d_result)
      e = cudaMemcpyAsync(r->d_result, (char *)sl.d_out + r->dev_off, row,
                          cudaMemcpyDeviceToDevice, ln.copy);
    if (e != cudaSuccess) st = APSPIE_ERR_CUDA;
  }
  cudaEventRecord(g.end, ln.copy);
  return st;
}

// Builds the groups of a batch on slot sl and launches them, cheapest first.
void launch_slot(apspie_server *s, Slot &sl, std::vector<Request *> batch) {
  {
    std::lock_guard<std::mutex> lock(s->mu);
    // The main lane leaves a quarter of the GPU to the deep lane while deep
    // traversals are in this batch or still running in the other slot;
    // otherwise it takes the whole GPU (a lone query at a low rate then runs
    // as fast as on the plain path).  A full-grid launch queued behind a
    // running deep traversal starts once that ends.
    bool deep = false;
    for (Request *r : batch)
      if (r->type != 2 && s->graphs[r->graph].deep) deep = true;
    for (Slot &o : s->slots)
      if (&o != &sl && o.busy)
        for (Group &g : o.groups)
          if (!g.done && g.lane == 1) deep = true;
    int resident = 0;
    apspie_ctx_resident_blocks(sl.lane[0].ctx, &resident);
    apspie_ctx_set_max_grid(sl.lane[0].ctx, deep ? std::max(1, resident - resident / 4) : 0);
  }
  // the groups, their order and their rows read the graph table: under the
  // lock, since another thread may add a graph meanwhile
  std::unique_lock<std::mutex> table_lock(s->mu);
  std::map<std::pair<int, int>, size_t> index;
  std::map<std::pair<int, uint32_t>, size_t> mis_index;
  sl.groups.clear();
  for (Request *r : batch) {
    if (r->type == 2) {
      // MIS queries of one graph and seed are the same query: one group
      auto key = std::make_pair(r->graph, r->seed);
      auto it = mis_index.find(key);
      if (it != mis_index.end()) {
        sl.groups[it->second].reqs.push_back(r);
        continue;
      }
      mis_index[key] = sl.groups.size();
      sl.groups.emplace_back();
      sl.groups.back().kind = 2;
      sl.groups.back().graph = r->graph;
      sl.groups.back().reqs.push_back(r);
      continue;
    }
    // A group holds at most one multi-source launch's worth of sources
    // (64 BFS / 32 SSSP), the size every lane was warmed with: a larger one
    // would run as several device jobs in one launch and need more
    // workspace than the warm-up gave, and growing a workspace waits for
    // all device work.  The next query of the pair starts a new group.
    const size_t cap = s->graphs[r->graph].deep ? SIZE_MAX : (r->type == 0 ? 64u : 32u);
    auto key = std::make_pair(r->graph, r->type);
    auto it = index.find(key);
    if (it == index.end() || sl.groups[it->second].reqs.size() >= cap) {
      index[key] = sl.groups.size();
      sl.groups.emplace_back();
      sl.groups.back().kind = r->type;
      sl.groups.back().graph = r->graph;
      sl.groups.back().reqs.push_back(r);
    } else {
      sl.groups[it->second].reqs.push_back(r);
    }
  }
  for (Group &g : sl.groups) g.lane = (s->graphs[g.graph].deep && g.kind != 2) ? 1 : 0;
  std::stable_sort(sl.groups.begin(), sl.groups.end(), [&](const Group &a, const Group &b) {
    return s->graphs[a.graph].cost_ms[a.kind] < s->graphs[b.graph].cost_ms[b.kind];
  });
  // rows: a group's results are consecutive (a batch job writes [nsrc][m])
  // (replayed results that only have to reach host memory all land on the
  // same staging row: the copy is what is measured, not the bytes kept)
  size_t dev = 0, host = 0, sink = 0;
  for (Group &g : sl.groups)
    for (Request *r : g.reqs) {
      const size_t row = 4 * (size_t)s->graphs[r->graph].m;
      r->dev_off = dev;
      dev += row;
      if (r->h_result) {
        r->host_off = host;
        host += row;
      } else if (r->to_stage) {
        sink = std::max(sink, row);
      }
    }
  for (Group &g : sl.groups)
    for (Request *r : g.reqs)
      if (!r->h_result && r->to_stage) r->host_off = host;
  host += sink;
  table_lock.unlock();
  while (sl.events.size() < 3 * sl.groups.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    sl.events.push_back(e);
  }
  const bool buffers =
      sl.events.size() >= 3 * sl.groups.size() &&
      ensure_buffer((void **)&sl.d_out, &sl.d_bytes, dev, false, &s->retired) &&
      (host == 0 || ensure_buffer(&sl.h_stage, &sl.h_bytes, host, true, &s->retired_host));
  for (size_t i = 0; i < sl.groups.size(); ++i) {
    Group &g = sl.groups[i];
    if (!buffers) {
      g.status = APSPIE_ERR_OOM;
      continue;
    }
    g.start = sl.events[3 * i];
    g.end = sl.events[3 * i + 1];
    g.computed = sl.events[3 * i + 2];
    g.status = launch_group(s, sl, g);
  }
  if (!buffers) {
    // nothing was launched: complete the groups with the error
    for (Group &g : sl.groups) {
      g.start = g.end = nullptr;
      std::lock_guard<std::mutex> lock(s->mu);
      for (Request *r : g.reqs) {
        r->status = APSPIE_ERR_OOM;
        r->done = true;
        s->in_flight -= r->bytes;
        ++s->completed;
      }
      g.done = true;
    }
    s->cv.notify_all();
    sl.groups.clear();
    return;
  }
  sl.busy = true;
}

// The worker's pause between polls of the running groups' events (every
// slot is polled at the top of its loop, so a finished group is reported
// within about this long whichever slot it is in).
void pause_briefly() { std::this_thread::sleep_for(std::chrono::microseconds(20)); }

void worker_main(apspie_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    for (Slot &sl : s->slots)
      if (sl.busy) poll_slot(s, sl, false);
    Slot *free_slot = nullptr;
    for (Slot &sl : s->slots)
      if (!sl.busy) free_slot = &sl;
    if (!free_slot) {
      // both batches in flight: poll again shortly.  Waiting on one slot's
      // group instead left the other slot's finished groups unreported
      // until that group ended (bursts of 100 - 400 ms latency at 100 q/s).
      pause_briefly();
      continue;
    }
    // One slot free, the other running: while its main lane still has two
    // or more groups queued the GPU has work, so the next batch waits and
    // gathers the queries that arrive meanwhile (larger groups share more
    // of each traversal); it forms once the last main-lane group runs.
    Group *queued = nullptr;
    for (Slot &sl : s->slots) {
      if (!sl.busy) continue;
      int left = 0;
      for (Group &g : sl.groups)
        if (!g.done && g.lane == 0 && g.end) {
          if (!queued) queued = &g;
          ++left;
        }
      if (left < 2) queued = nullptr;
      if (queued) break;
    }
    if (queued) {
      pause_briefly();
      continue;
    }
    std::vector<Request *> batch;
    {
      std::unique_lock<std::mutex> lock(s->mu);
      const bool any_busy = s->slots[0].busy || s->slots[1].busy;
      if (s->stop && s->pending.empty() && !any_busy) return;
      if (s->pending.empty() || s->warming) {
        s->cv.wait_for(lock, std::chrono::microseconds(any_busy ? 20 : 2000));
        continue;
      }
      // admit in arrival order while the state budget and the device's
      // free memory (less a reserve for the library's own buffers) allow
      refresh_free_locked(s);
      const size_t cap = s->free_known ? std::min(s->budget, s->mem_cap) : s->budget;
      while (!s->pending.empty() && (int)batch.size() < s->max_batch) {
        Request *r = s->pending.front();
        const bool first = s->in_flight == 0 && batch.empty();
        if (!first && s->in_flight + r->bytes > cap) {
          ++s->mem_waits;
          break;
        }
        s->pending.pop_front();
        s->in_flight += r->bytes;
        batch.push_back(r);
      }
    }
    if (batch.empty()) {
      // over budget: poll again shortly, until a running group releases
      // its memory
      pause_briefly();
      continue;
    }
    const auto t_launch = Clock::now();
    launch_slot(s, *free_slot, std::move(batch));
    const double launch_ms =
        std::chrono::duration<double, std::milli>(Clock::now() - t_launch).count();
    {
      std::lock_guard<std::mutex> lock(s->mu);
      s->max_launch_ms = std::max(s->max_launch_ms, launch_ms);
      ++s->batches;
    }
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
  for (Slot &sl : s->slots)
    for (int l = 0; l < 2; ++l) {
      Lane &ln = sl.lane[l];
      if (cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaStreamCreateWithFlags(&ln.copy, cudaStreamNonBlocking) != cudaSuccess ||
          apspie_ctx_create(device, ln.stream, &ln.ctx) != APSPIE_OK) {
        cudaGetLastError();
        apspie_server_destroy(s);
        return APSPIE_ERR_CUDA;
      }
      if (l == 1) {
        // the deep lane: a quarter of the resident persistent blocks (its
        // traversals are latency bound per level; the main lane's large
        // graphs need the blocks)
        int resident = 0;
        apspie_ctx_resident_blocks(ln.ctx, &resident);
        apspie_ctx_set_max_grid(ln.ctx, std::max(1, resident / 4));
      }
    }
  try {
    s->worker = std::thread(worker_main, s);
  } catch (const std::exception &) {  // no thread could be started
    apspie_server_destroy(s);
    return APSPIE_ERR_OOM;
  }
  *out = s;
  return APSPIE_OK;
}

}  // extern "C"

namespace {

// The first query of a graph on a lane grows that lane's workspaces (and,
// for a deep graph, creates its sub-contexts: one stream and workspace per
// concurrent single-source traversal, up to 48); growing frees the old
// buffer, which synchronises the device, and the first queries took
// hundreds of ms.  A new graph is therefore run once on every lane that
// will serve it, at add time: one query of each kind alone and the largest
// groups (64 BFS, 32 SSSP sources; 48 each on a deep graph) -- only while
// the server is idle, since a context serves one thread at a time.
void warm_lanes(apspie_server *s, const GraphEntry &g) {
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->in_flight != 0 || !s->pending.empty() || s->slots[0].busy || s->slots[1].busy)
      return;
    s->warming = true;
  }
  const int kb = g.deep ? 48 : 64, ks = g.deep ? 48 : 32;
  int32_t *out = nullptr;
  uint32_t *prio = nullptr;
  if (cudaMalloc(&out, sizeof(int32_t) * (size_t)g.m * kb) == cudaSuccess &&
      cudaMalloc(&prio, sizeof(uint32_t) * (size_t)g.m) == cudaSuccess &&
      cudaMemset(prio, 0, sizeof(uint32_t) * (size_t)g.m) == cudaSuccess) {
    std::vector<int> src(kb);
    for (int i = 0; i < kb; ++i) src[i] = (int)((int64_t)g.m * i / kb);
    apspie_job jobs[2];
    int nj = 0;
    for (int kind = 0; kind < 2; ++kind) {
      if (kind == 1 && !g.w) break;
      apspie_job &j = jobs[nj++];
      std::memset(&j, 0, sizeof(j));
      j.type = kind == 0 ? APSPIE_JOB_BFS : APSPIE_JOB_SSSP_U32;
      j.m = g.m;
      j.nnz = g.nnz;
      j.d_ptr = g.ptr;
      j.d_ind = g.ind;
      j.d_tptr = g.tptr;
      j.d_tind = g.tind;
      j.d_w = g.w;
      j.symmetric = g.symmetric;
      j.nsrc = kind == 0 ? kb : ks;
      j.h_src = src.data();
      j.d_out = out;
      j.alpha = j.beta = -1;
    }
    const int *tp = g.tptr ? g.tptr : (g.symmetric ? g.ptr : nullptr);
    const int *ti = g.tptr ? g.tind : (g.symmetric ? g.ind : nullptr);
    for (Slot &sl : s->slots) {
      Lane &ln = sl.lane[g.deep ? 1 : 0];
      apspie_bfs(ln.ctx, src[0], g.nnz, g.m, g.ptr, g.ind, tp, ti, out, 0);
      if (g.w) sssp_one(ln.ctx, g, src[0], (uint32_t *)out);
      if (g.symmetric) apspie_mis(ln.ctx, g.nnz, g.m, g.ptr, g.ind, prio, out, 1.0f);
      for (int i = 0; i < nj; ++i)
        if (apspie_batch_run(ln.ctx, 1, &jobs[i], 0) != APSPIE_OK) break;
      apspie_ctx_sync(ln.ctx);
    }
  }
  cudaFree(out);
  cudaFree(prio);
  cudaGetLastError();
  std::lock_guard<std::mutex> lock(s->mu);
  s->warming = false;
  s->cv.notify_all();
}

}  // namespace

extern "C" {

int apspie_server_add_graph(apspie_server_t s, int m, int64_t nnz, const int *d_ptr,
                            const int *d_ind, const int *d_tptr, const int *d_tind,
                            const uint32_t *d_w, int symmetric, int *graph_id) {
  if (!s || m <= 0 || nnz < 0 || !d_ptr || (nnz > 0 && !d_ind) || !graph_id)
    return APSPIE_ERR_INVALID;
  GraphEntry g{m, nnz, d_ptr, d_ind, d_tptr, d_tind, d_w, symmetric, false, {0, 0, 0}};
  g.stptr = nullptr;
  int levels = 0;
  int st = probe_levels(s->device, g, &levels);
  if (st != APSPIE_OK) return st;
  g.deep = levels > kDeepLevels;
  // first guesses of a group's device time, replaced by measurements
  g.cost_ms[0] = 1e-6f * (float)nnz * (g.deep ? 100.0f : 1.0f);
  g.cost_ms[1] = 4.0f * g.cost_ms[0];
  g.cost_ms[2] = 2.0f * g.cost_ms[0];
  try {
    warm_lanes(s, g);
  } catch (const std::exception &) {  // the warm-up is an optimisation only
    std::lock_guard<std::mutex> lock(s->mu);
    s->warming = false;
    s->cv.notify_all();
  }
  std::lock_guard<std::mutex> lock(s->mu);
  try {
    s->graphs.push_back(g);
  } catch (const std::bad_alloc &) {
    return APSPIE_ERR_OOM;
  }
  if (g.deep) s->any_deep = true;
  *graph_id = (int)s->graphs.size() - 1;
  return APSPIE_OK;
}

int apspie_server_set_sssp_in(apspie_server_t s, int graph, const int *d_tptr,
                              const int *d_tind, const uint32_t *d_tw) {
  if (!s || !d_tptr) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  if (graph < 0 || graph >= (int)s->graphs.size()) return APSPIE_ERR_INVALID;
  GraphEntry &g = s->graphs[graph];
  if (g.nnz > 0 && (!d_tind || !d_tw)) return APSPIE_ERR_INVALID;
  g.stptr = d_tptr;
  g.stind = d_tind;
  g.stw = d_tw;
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
  try {  // into the table, then the queue; undone if either cannot grow
    s->reqs[r->id] = r;
    try {
      s->pending.push_back(r);
    } catch (...) {
      s->reqs.erase(r->id);
      throw;
    }
  } catch (const std::bad_alloc &) {
    delete r;
    return APSPIE_ERR_OOM;
  }
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

int apspie_server_replay(apspie_server_t s, int n, const apspie_query *q, int to_host,
                         double *lat_ms, double *wall_ms) {
  return apspie_server_replay_keep(s, n, q, to_host, nullptr, lat_ms, wall_ms);
}

int apspie_server_replay_keep(apspie_server_t s, int n, const apspie_query *q, int to_host,
                              int32_t *const *d_keep, double *lat_ms, double *wall_ms) {
  if (!s || n < 0 || (n > 0 && (!q || !lat_ms))) return APSPIE_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (int i = 0; i < n; ++i)
      if (check_query(s, q[i].type, q[i].graph, q[i].source) || q[i].t_us < 0 ||
          (i > 0 && q[i].t_us < q[i - 1].t_us))
        return APSPIE_ERR_INVALID;
  }
  std::vector<Request *> rs;
  try {
    rs.assign((size_t)n, nullptr);
  } catch (const std::bad_alloc &) {
    return APSPIE_ERR_OOM;
  }
  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(1);
  int st = APSPIE_OK;
  for (int i = 0; i < n && st == APSPIE_OK; ++i) {
    const Clock::time_point at =
        t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(q[i].t_us));
    spin_until(at);
    std::lock_guard<std::mutex> lock(s->mu);
    // the pending queue is large; a full one is waited out, the query keeps
    // its scheduled arrival time
    int32_t *keep = d_keep ? d_keep[i] : nullptr;
    while ((st = enqueue_locked(s, q[i].type, q[i].graph, q[i].source, q[i].seed, nullptr, keep,
                                at, &rs[i])) == APSPIE_ERR_BUSY) {
      s->mu.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(100));
      s->mu.lock();
    }
    if (st == APSPIE_OK) rs[i]->to_stage = to_host != 0;
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

int apspie_server_replay_plain(apspie_server_t s, int n, const apspie_query *q, int to_host,
                               double *lat_ms, double *wall_ms) {
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
  int st = APSPIE_OK;
  if (!s->plain_ctx) {
    if (cudaStreamCreateWithFlags(&s->plain_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      s->plain_stream = nullptr;
      return APSPIE_ERR_CUDA;
    }
    st = apspie_ctx_create(s->device, s->plain_stream, &s->plain_ctx);
    if (st != APSPIE_OK) return st;
  }
  if (s->plain_m < (size_t)std::max(maxm, 1)) {
    cudaFree(s->plain_row);
    if (s->plain_hrow) cudaFreeHost(s->plain_hrow);
    s->plain_row = nullptr;
    s->plain_hrow = nullptr;
    s->plain_m = 0;
    const size_t mm = (size_t)std::max(maxm, 1);
    if (cudaMalloc(&s->plain_row, 4 * mm) != cudaSuccess ||
        cudaMallocHost(&s->plain_hrow, 4 * mm) != cudaSuccess) {
      cudaGetLastError();
      return APSPIE_ERR_OOM;
    }
    s->plain_m = mm;
  }
  cudaStream_t stream = s->plain_stream;
  apspie_ctx ctx = s->plain_ctx;
  int32_t *row = s->plain_row;
  void *h_row = s->plain_hrow;
  const Clock::time_point t0 = Clock::now() + std::chrono::milliseconds(1);
  double last = 0;
  for (int i = 0; i < n && st == APSPIE_OK; ++i) {
    const Clock::time_point at =
        t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(q[i].t_us));
    spin_until(at);  // returns at once when the previous query ran late
    GraphEntry g;
    {
      std::lock_guard<std::mutex> lock(s->mu);  // the table may grow meanwhile
      g = s->graphs[q[i].graph];
    }
    if (q[i].type == 0) {
      const int *tp = g.symmetric ? g.ptr : g.tptr, *ti = g.symmetric ? g.ind : g.tind;
      st = apspie_bfs(ctx, q[i].source, g.nnz, g.m, g.ptr, g.ind, tp, ti, row, 0);
    } else if (q[i].type == 1) {
      st = sssp_one(ctx, g, q[i].source, (uint32_t *)row);
    } else {
      uint32_t *prio = nullptr;
      st = get_prio(s, q[i].graph, (size_t)g.m, q[i].seed, stream, &prio);
      if (st == APSPIE_OK) st = apspie_mis(ctx, g.nnz, g.m, g.ptr, g.ind, prio, row, 1.0f);
    }
    if (st == APSPIE_OK && to_host &&
        cudaMemcpyAsync(h_row, row, 4 * (size_t)g.m, cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      st = APSPIE_ERR_CUDA;
    if (st == APSPIE_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = APSPIE_ERR_CUDA;
    const double l = std::chrono::duration<double, std::milli>(Clock::now() - at).count();
    lat_ms[i] = l;
    last = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
  if (wall_ms) *wall_ms = last;
  return st;
}

int apspie_server_debug_fail_next(apspie_server_t s, int kind) {
  if (!s || kind < 0 || kind > 2) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  s->fail_next_kind = kind;
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
  std::vector<double> l;
  try {
    l = s->latencies;
  } catch (const std::bad_alloc &) {
    return APSPIE_ERR_OOM;
  }
  std::sort(l.begin(), l.end());
  auto q = [&](double p) {
    if (l.empty()) return 0.0;
    size_t i = (size_t)std::min<double>((double)l.size() - 1, p * (double)(l.size() - 1) + 0.5);
    return l[i];
  };
  out->p50_ms = q(0.50);
  out->p99_ms = q(0.99);
  out->max_ms = l.empty() ? 0.0 : l.back();
  out->admission_waits = s->mem_waits;
  out->memory_cap_bytes = s->mem_cap;
  out->max_launch_ms = s->max_launch_ms;
  return APSPIE_OK;
}

int apspie_server_reset_stats(apspie_server_t s) {
  if (!s) return APSPIE_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  s->latencies.clear();
  s->completed = 0;
  s->batches = 0;
  s->launched_jobs = 0;
  s->mem_waits = 0;
  s->max_launch_ms = 0.0;
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
    for (Lane &ln : sl.lane) {
      if (ln.stream) cudaStreamSynchronize(ln.stream);
      if (ln.copy) cudaStreamSynchronize(ln.copy);
      if (ln.ctx) apspie_ctx_destroy(ln.ctx);
      if (ln.stream) cudaStreamDestroy(ln.stream);
      if (ln.copy) cudaStreamDestroy(ln.copy);
    }
    for (cudaEvent_t e : sl.events) cudaEventDestroy(e);
    cudaFree(sl.d_out);
    if (sl.h_stage) cudaFreeHost(sl.h_stage);
  }
  if (s->plain_ctx) apspie_ctx_destroy(s->plain_ctx);
  if (s->plain_stream) cudaStreamDestroy(s->plain_stream);
  cudaFree(s->plain_row);
  if (s->plain_hrow) cudaFreeHost(s->plain_hrow);
  for (void *q : s->retired) cudaFree(q);
  for (void *q : s->retired_host) cudaFreeHost(q);
  for (auto &kv : s->prio_cache) cudaFree(kv.second);
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
  return APSPIE_OK;
}

}  // extern "C"
