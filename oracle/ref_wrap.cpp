// ref_wrap.cpp -- C entry points around the reference's own CPU routines.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile from the reference
// sources where they lie (src/testBfs.cpp, src/testSssp.cpp with its Boost
// lines stripped, src/mt19937ar.cpp) into oracle/_ref/libapspie_ref.so.  No
// reference source is copied into this repository; the stripped SSSP file is
// a build intermediate that the recipe deletes after compiling.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/time.h>
#include <vector>

// The reference's drivers take CpuTimer and print_array from src/util.cuh,
// which needs the CUDA toolkit and moderngpu; these host-only stand-ins
// provide the two members the CPU routines use.
struct CpuTimer {
  double s = 0, e = 0;
  void Start() { timeval t; gettimeofday(&t, 0); s = t.tv_sec + 1e-6 * t.tv_usec; }
  void Stop() { timeval t; gettimeofday(&t, 0); e = t.tv_sec + 1e-6 * t.tv_usec; }
  float ElapsedMillis() { return (float)(1000.0 * (e - s)); }
};
template <typename T> void print_array(T *, int) {}

#include "testBfs.cpp"             // src/testBfs.cpp:7-90
#include "testSssp_noboost.inc"    // src/testSssp.cpp:1-133 minus lines 3-7, 11
#include "mt19937ar.h"             // src/mt19937ar.h

extern "C" {

// bfsCPU (src/testBfs.cpp:75-90).  Returns the search depth.
int ref_bfs_cpu(int src, int m, const int *rowptr, const int *colind,
                int *depth, int stop) {
  return bfsCPU<int>(src, m, rowptr, colind, depth, stop);
}

// ssspCPU (src/testSssp.cpp:117-133).  SimpleReferenceSssp reads
// h_csrValA[i] for every vertex i < m while seeding its queue
// (src/testSssp.cpp:52-55), so the weights are padded to max(nnz, m).
int ref_sssp_cpu(int src, int m, const int *rowptr, const int *colind,
                 const float *w, float *dist, int stop) {
  int nnz = rowptr[m];
  std::vector<float> wp((size_t)(nnz > m ? nnz : m) + 1, 1.0f);
  if (nnz) std::memcpy(wp.data(), w, sizeof(float) * (size_t)nnz);
  return ssspCPU(src, m, rowptr, colind, wp.data(), dist, stop);
}

// init_genrand + genrand_int32 (src/mt19937ar.cpp:57-150).
void ref_mt_fill(unsigned long seed, long long n, unsigned int *out) {
  init_genrand(seed);
  for (long long i = 0; i < n; ++i) out[i] = (unsigned int)genrand_int32();
}
}
