// ref_kernels.cpp -- host builds of the reference's own TC and MIS kernels.
//
// TEST INFRASTRUCTURE ONLY.  The reference's triangle-count intersection
// ewiseMultTc (src/tc.cuh:168-199) and its MIS round kernels (diff,
// preprocessFlag, streamCompact, scatterFloat, gather, buildVector,
// updateMis, updateNeighbor: src/spmspvMis.cuh:10-78) are plain
// per-element loops over grid-stride indices with no library code inside.
// oracle/Makefile extracts those line ranges into build intermediates
// (deleted after compiling) that are included below with __global__ removed
// and the CUDA built-in index variables provided as host globals, so the
// reference's own loop bodies run on the CPU.  Launches are emulated by
// iterating blockIdx / threadIdx over the grid the reference launches.
//
// The library calls between those kernels in the reference's MIS loop
// (mgpu::Scan, IntervalGather / IntervalExpand, cub::DeviceRadixSort::
// SortPairs, mgpu::ReduceByKey with maximum; src/spmspvMis.cuh:248-289)
// live in absent third-party code and are restated here as plain loops with
// their documented semantics (exclusive scan, gather of the frontier's
// neighbour lists in frontier order, stable sort of (key, value) pairs by
// key, per-key maximum).  The triangle-count product U*L that feeds
// ewiseMultTc comes from the caller (cuSPARSE csrgemm in the reference).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace refk {

struct HostDim3 {
  unsigned x, y, z;
};
static HostDim3 gridDim = {1, 1, 1}, blockDim = {1, 1, 1};
static HostDim3 blockIdx = {0, 0, 0}, threadIdx = {0, 0, 0};

#define __global__
#include "misKernels.inc"   // src/spmspvMis.cuh:10-78
#include "ewiseMultTc.inc"  // src/tc.cuh:168-199
#undef __global__

// One host thread covers every index of a grid-stride kernel.
template <typename F>
static void launch_serial(F f) {
  gridDim = {1, 1, 1};
  blockDim = {1, 1, 1};
  blockIdx = {0, 0, 0};
  threadIdx = {0, 0, 0};
  f();
}

}  // namespace refk

extern "C" {

// ewiseMultTc<T> (src/tc.cuh:168-199) launched as test/tc/main.cu:244 does:
// NB = ceil(m / 512) blocks of NT = 512 threads, thread tid handling column
// tid.  D (the product U*L) and C (the strictly upper part) are CSC with m + 1
// column offsets; their row index arrays must hold one readable entry past
// the last column (the kernel reads d_cscRowInd*[i] after i reaches the
// column end, src/tc.cuh:190,194).  out receives NB * NT per-thread counts
// (entries >= m are 0); T = double.
void ref_tc_ewise(int m, int64_t nnzD, const double *valD, const int *ptrD, const int *indD,
                  const double *valC, const int *ptrC, const int *indC, double *out) {
  const int NT = 512;
  const int NB = (m + NT - 1) / NT;
  for (int b = 0; b < NB; ++b)
    for (int t = 0; t < NT; ++t) {
      refk::gridDim = {(unsigned)NB, 1, 1};
      refk::blockDim = {(unsigned)NT, 1, 1};
      refk::blockIdx = {(unsigned)b, 0, 0};
      refk::threadIdx = {(unsigned)t, 0, 0};
      refk::ewiseMultTc<double>((int)nnzD, m, valD, ptrD, indD, valC, ptrC, indC, out);
    }
}

// The round loop of spmspvMis (src/spmspvMis.cuh:232-318) over the
// reference's kernels, typeVal = double.  prio: m priorities; result: m
// entries (1 in the set, 0 out, -1 undecided).  Returns the rounds that
// processed a frontier.
int ref_mis(int m, const int *ptr, const int *ind, const double *prio, float delta, int *mis) {
  using namespace refk;
  std::vector<int> rowdiff(m), x(m), good((size_t)m + 1), keys, vals, keys_alt;
  std::vector<double> temp(m), vecval, swapval;
  for (int i = 0; i < m; ++i) mis[i] = -1;
  launch_serial([&] { diff(ptr, rowdiff.data(), m); });
  float minimum = 1;
  int rounds = 0;
  for (int iter = 1; iter < 150; ++iter) {
    if (minimum >= 0) minimum -= delta;
    launch_serial([&] { buildVector<double>(m, minimum, prio, mis, x.data()); });
    // mgpu::Scan exclusive: good[i] = sum x[0..i), count = sum x
    int count = 0;
    for (int i = 0; i < m; ++i) {
      good[i] = count;
      count += x[i];
    }
    if (count > 0) {
      ++rounds;
      std::vector<int> front(count);
      launch_serial([&] { streamCompact(x.data(), good.data(), front.data(), m); });
      // IntervalGather / IntervalExpand: for each frontier vertex u in
      // order, its neighbour list; key = neighbour, value = u
      keys.clear();
      vals.clear();
      for (int u : front)
        for (int k = ptr[u]; k < ptr[u + 1]; ++k) {
          keys.push_back(ind[k]);
          vals.push_back(u);
        }
      const int total = (int)keys.size();
      launch_serial([&] { preprocessFlag<double>(temp.data(), m); });
      // cub::DeviceRadixSort::SortPairs: stable by key
      std::vector<int> order(total);
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(),
                       [&](int a, int b) { return keys[a] < keys[b]; });
      std::vector<int> sk(total), sv(total);
      for (int i = 0; i < total; ++i) {
        sk[i] = keys[order[i]];
        sv[i] = vals[order[i]];
      }
      keys.swap(sk);
      vals.swap(sv);
      vecval.assign((size_t)total + 1, 0.0);
      launch_serial([&] { gather<double>(total, vals.data(), prio, vecval.data()); });
      // ReduceByKey(maximum) over equal adjacent keys
      keys_alt.clear();
      swapval.clear();
      for (int i = 0; i < total;) {
        int j = i;
        double best = vecval[i];
        while (j < total && keys[j] == keys[i]) {
          best = std::max(best, vecval[j]);
          ++j;
        }
        keys_alt.push_back(keys[i]);
        swapval.push_back(best);
        i = j;
      }
      const int nred = (int)keys_alt.size();
      launch_serial(
          [&] { scatterFloat<double>(nred, keys_alt.data(), swapval.data(), temp.data()); });
      launch_serial([&] { updateMis<double>(m, mis, temp.data(), prio, x.data()); });
      launch_serial([&] {
        updateNeighbor<double>(total, mis, keys.data(), vals.data(), vecval.data(), prio);
      });
    } else if (minimum <= (float)0) {
      break;
    }
  }
  return rounds;
}

}  // extern "C"
