// ref_api_main.cpp -- a test driver written against the reference's API.
//
// Mirrors the reference's test/<algo>/main.cu drivers: read a Matrix Market
// file, build the CSR with buildMatrix, run the CPU oracle, run the GPU
// routine through the reference's signatures (include/apspie_ref.hpp), then
// verify() / unverify().  Exit status 0 means CORRECT.
//
//   ref_api_main <bfs|spmspvbfs|sssp|mis|mxv|spmv|csr2csc|spgemm|spgemm_csc|mxm|tc> file.mtx
//                [-source N] [-undirected]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "apspie_ref.hpp"
#include "oracle.h"

namespace {

struct HostCsr {
  int m = 0;
  int64_t nnz = 0;
  std::vector<int> ptr, ind;
  std::vector<float> val;
};

HostCsr read(const char *path, bool undirected) {
  HostCsr g;
  int *p = nullptr, *i = nullptr, weighted = 0;
  float *v = nullptr;
  apspie::check(apspie_read_mtx_host(path, undirected, &g.m, &g.nnz, &p, &i, &v, &weighted),
                nullptr, "read_mtx");
  g.ptr.assign(p, p + g.m + 1);
  g.ind.assign(i, i + g.nnz);
  g.val.assign(v, v + g.nnz);
  apspie_host_free(p);
  apspie_host_free(i);
  apspie_host_free(v);
  if (!weighted)
    for (int64_t k = 0; k < g.nnz; ++k) g.val[k] = 1.0f + (float)((k * 37) % 11);
  return g;
}

// COO (row, col, val) of a CSR, as the reference drivers hold before buildMatrix
void to_coo(const HostCsr &g, std::vector<int> &r, std::vector<int> &c, std::vector<float> &v) {
  for (int u = 0; u < g.m; ++u)
    for (int k = g.ptr[u]; k < g.ptr[u + 1]; ++k) {
      r.push_back(u);
      c.push_back(g.ind[k]);
      v.push_back(g.val[k]);
    }
}

template <typename T>
std::vector<T> download(const T *d, size_t n) {
  std::vector<T> h(n);
  cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost);
  return h;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    printf("Usage: %s algo file.mtx [-source N] [-undirected]\n", argv[0]);
    return 2;
  }
  std::string algo = argv[1];
  int source = 0;
  bool undirected = false;
  for (int a = 3; a < argc; ++a) {
    if (!strcmp(argv[a], "-source") && a + 1 < argc) source = atoi(argv[++a]);
    else if (!strcmp(argv[a], "-undirected")) undirected = true;
  }
  HostCsr g = read(argv[2], undirected);
  const int m = g.m, edge = (int)g.nnz;
  printf("Testing %s on %s from source %d: %d nodes, %d edges\n", algo.c_str(), argv[2], source, m,
         edge);
  mgpu::ContextPtr context = mgpu::CreateCudaDevice(0);
  context->SetUndirected(undirected);

  std::vector<int> rows, cols;
  std::vector<float> vals;
  to_coo(g, rows, cols, vals);
  d_matrix A;
  matrix_new(&A, m, m);
  buildMatrix<float>(&A, edge, rows.data(), cols.data(), vals.data());

  int errors = 0;
  try {
    if (algo == "bfs" || algo == "spmspvbfs") {
      int *d_bfs = nullptr;
      cudaMalloc(&d_bfs, sizeof(int) * m);
      std::vector<int> cpu(m);
      int depth = orc_bfs(m, g.ptr.data(), g.ind.data(), source, 1 << 30, cpu.data());
      if (algo == "bfs")
        bfs<int>(source, edge, m, A.h_cscColPtr, A.d_cscColPtr, A.d_cscRowInd, d_bfs, depth,
                 *context);
      else
        spmspvBfs(source, edge, m, A.h_cscColPtr, A.d_cscColPtr, A.d_cscRowInd, d_bfs, depth,
                  *context);
      errors = verify(m, download(d_bfs, m).data(), cpu.data());
      cudaFree(d_bfs);
    } else if (algo == "sssp") {
      float *d_dist = nullptr;
      cudaMalloc(&d_dist, sizeof(float) * m);
      std::vector<float> cpu(m);
      orc_sssp_f32(m, g.ptr.data(), g.ind.data(), g.val.data(), source, cpu.data());
      sssp<float>(source, edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_dist, 1000,
                  *context);
      errors = verify(m, download(d_dist, m).data(), cpu.data());
      cudaFree(d_dist);
    } else if (algo == "mis") {
      std::vector<uint32_t> prio(m);
      apspie_mt19937_fill_host(5489u, m, prio.data());
      uint32_t *d_prio = nullptr;
      int *d_mis = nullptr, *d_flags = nullptr;
      cudaMalloc(&d_prio, sizeof(uint32_t) * m);
      cudaMalloc(&d_mis, sizeof(int) * m);
      cudaMalloc(&d_flags, sizeof(int) * m);
      cudaMemcpy(d_prio, prio.data(), sizeof(uint32_t) * m, cudaMemcpyHostToDevice);
      spmspvMis<uint32_t>(edge, m, A.h_cscColPtr, A.d_cscColPtr, A.d_cscRowInd, d_prio, d_mis,
                          0.1f, *context);
      // the reference's check: neighbour flags + membership == 1
      spmspvCsr<int>(d_mis, edge, m, A.d_cscColPtr, A.d_cscRowInd, d_flags, *context);
      std::vector<int> h_mis = download(d_mis, m), h_flags = download(d_flags, m);
      errors = unverify(m, h_flags.data(), h_mis.data());
      std::vector<int> cpu(m);
      orc_mis(m, g.ptr.data(), g.ind.data(), prio.data(), cpu.data());
      errors += verify(m, h_mis.data(), cpu.data());
      cudaFree(d_prio);
      cudaFree(d_mis);
      cudaFree(d_flags);
    } else if (algo == "mxv") {
      // dense mXv with a one-hot frontier: y = A^T e_source as in one BFS level
      std::vector<float> x(m, 0.0f);
      x[source] = 1.0f;
      float *d_x = nullptr, *d_y = nullptr;
      cudaMalloc(&d_x, sizeof(float) * m);
      cudaMalloc(&d_y, sizeof(float) * m);
      cudaMemcpy(d_x, x.data(), sizeof(float) * m, cudaMemcpyHostToDevice);
      d_scratch *d;
      allocScratch(&d, edge, m);
      int total = mXv<float>(d_x, edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_y, d,
                             *context);
      std::vector<float> expect(m, 0.0f);
      for (int k = g.ptr[source]; k < g.ptr[source + 1]; ++k) expect[g.ind[k]] += g.val[k];
      errors = verify(m, download(d_y, m).data(), expect.data());
      errors += total != g.ptr[source + 1] - g.ptr[source];
      delete d;
      cudaFree(d_x);
      cudaFree(d_y);
    } else if (algo == "spmv") {
      // dense SpMV over every row: y = A x, x[j] = j + 1
      std::vector<float> x(m);
      for (int j = 0; j < m; ++j) x[j] = (float)(j + 1);
      float *d_x = nullptr, *d_y = nullptr;
      cudaMalloc(&d_x, sizeof(float) * m);
      cudaMalloc(&d_y, sizeof(float) * m);
      cudaMemcpy(d_x, x.data(), sizeof(float) * m, cudaMemcpyHostToDevice);
      spmv<float>(d_x, edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_y, *context);
      std::vector<float> expect(m, 0.0f);
      for (int r = 0; r < m; ++r) {
        double acc = 0;
        for (int k = g.ptr[r]; k < g.ptr[r + 1]; ++k) acc += (double)g.val[k] * x[g.ind[k]];
        expect[r] = (float)acc;
      }
      errors = verify(m, download(d_y, m).data(), expect.data());
      cudaFree(d_x);
      cudaFree(d_y);
    } else if (algo == "csr2csc") {
      float *d_tv = nullptr;
      int *d_tp = nullptr, *d_ti = nullptr;
      cudaMalloc(&d_tv, sizeof(float) * (edge > 0 ? edge : 1));
      cudaMalloc(&d_ti, sizeof(int) * (edge > 0 ? edge : 1));
      cudaMalloc(&d_tp, sizeof(int) * (m + 1));
      csr2csc<float>(m, edge, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_tv, d_ti, d_tp,
                     *context);
      // host transpose: column-major counting sort of the same arrays
      std::vector<int> tp(m + 1, 0), ti(edge), fill;
      std::vector<float> tv(edge);
      for (int k = 0; k < edge; ++k) ++tp[g.ind[k] + 1];
      for (int j = 0; j < m; ++j) tp[j + 1] += tp[j];
      fill.assign(tp.begin(), tp.end() - 1);
      for (int r = 0; r < m; ++r)
        for (int k = g.ptr[r]; k < g.ptr[r + 1]; ++k) {
          ti[fill[g.ind[k]]] = r;
          tv[fill[g.ind[k]]++] = g.val[k];
        }
      errors = verify(m + 1, download(d_tp, m + 1).data(), tp.data());
      if (edge > 0) {
        errors += verify(edge, download(d_ti, edge).data(), ti.data());
        errors += verify(edge, download(d_tv, edge).data(), tv.data());
      }
      cudaFree(d_tv);
      cudaFree(d_ti);
      cudaFree(d_tp);
    } else if (algo == "spgemm") {
      d_matrix C;
      spgemm(&C, &A, &A, 0, 0, *context);
      std::vector<int64_t> cp(m + 1);
      int64_t nnz = orc_spgemm_symbolic(m, m, g.ptr.data(), g.ind.data(), g.ptr.data(),
                                        g.ind.data(), cp.data());
      std::vector<int> ci(nnz > 0 ? nnz : 1);
      std::vector<double> cv(nnz > 0 ? nnz : 1);
      orc_spgemm_numeric(m, m, g.ptr.data(), g.ind.data(), g.val.data(), g.ptr.data(),
                         g.ind.data(), g.val.data(), cp.data(), ci.data(), cv.data());
      std::vector<int> gptr = download(C.d_cscColPtr, m + 1);
      std::vector<int> gind = download(C.d_cscRowInd, (size_t)C.nnz);
      std::vector<float> gval = download(C.d_cscVal, (size_t)C.nnz);
      errors = (C.nnz != nnz);
      std::vector<int> cp32(cp.begin(), cp.end());
      errors += verify(m + 1, gptr.data(), cp32.data());
      if (!errors) {
        errors += verify((int)nnz, gind.data(), ci.data());
        std::vector<float> cvf(cv.begin(), cv.end());
        errors += verify((int)nnz, gval.data(), cvf.data());
      }
      matrix_delete(&C);
    } else if (algo == "spgemm_csc" || algo == "mxm") {
      // the reference's TC-driver SpGEMM (library-allocated C) and its
      // column-by-column mXm (caller's C), with B = the transpose of A so the
      // operand order shows: spgemm<T> forms A * B on the arrays, mXm B * A
      std::vector<int> tp(m + 1, 0), ti(g.nnz);
      std::vector<float> tv(g.nnz);
      for (int64_t k = 0; k < g.nnz; ++k) tp[g.ind[k] + 1]++;
      for (int v = 0; v < m; ++v) tp[v + 1] += tp[v];
      std::vector<int> at(tp.begin(), tp.end() - 1);
      for (int u = 0; u < m; ++u)
        for (int k = g.ptr[u]; k < g.ptr[u + 1]; ++k) {
          ti[at[g.ind[k]]] = u;
          tv[at[g.ind[k]]++] = 0.5f * g.val[k] + 1.0f;
        }
      int *d_tp = nullptr, *d_ti = nullptr;
      float *d_tv = nullptr;
      cudaMalloc(&d_tp, sizeof(int) * (m + 1));
      cudaMalloc(&d_ti, sizeof(int) * (g.nnz > 0 ? g.nnz : 1));
      cudaMalloc(&d_tv, sizeof(float) * (g.nnz > 0 ? g.nnz : 1));
      cudaMemcpy(d_tp, tp.data(), sizeof(int) * (m + 1), cudaMemcpyHostToDevice);
      cudaMemcpy(d_ti, ti.data(), sizeof(int) * g.nnz, cudaMemcpyHostToDevice);
      cudaMemcpy(d_tv, tv.data(), sizeof(float) * g.nnz, cudaMemcpyHostToDevice);
      const bool mxm = algo == "mxm";
      // the expected product, as CSR arrays: A * B (spgemm) or B * A (mXm)
      const int *lp = mxm ? tp.data() : g.ptr.data(), *li = mxm ? ti.data() : g.ind.data();
      const int *rp = mxm ? g.ptr.data() : tp.data(), *ri = mxm ? g.ind.data() : ti.data();
      const float *lv = mxm ? tv.data() : g.val.data(), *rv = mxm ? g.val.data() : tv.data();
      std::vector<int64_t> cp(m + 1);
      int64_t nnz = orc_spgemm_symbolic(m, m, lp, li, rp, ri, cp.data());
      std::vector<int> ci(nnz > 0 ? nnz : 1);
      std::vector<double> cv(nnz > 0 ? nnz : 1);
      orc_spgemm_numeric(m, m, lp, li, lv, rp, ri, rv, cp.data(), ci.data(), cv.data());
      int *d_cp = nullptr, *d_ci = nullptr;
      float *d_cv = nullptr;
      int got = 0;
      if (mxm) {
        cudaMalloc(&d_cp, sizeof(int) * (m + 1));
        cudaMalloc(&d_ci, sizeof(int) * 16 * (size_t)(edge > 0 ? edge : 1));
        cudaMalloc(&d_cv, sizeof(float) * 16 * (size_t)(edge > 0 ? edge : 1));
        got = mXm<float>(edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_tv, tp.data(), d_tp,
                         d_ti, d_cv, d_cp, d_ci, *context);
      } else {
        got = spgemm<float>(edge, m, A.d_cscVal, A.d_cscColPtr, A.d_cscRowInd, d_tv, d_tp, d_ti,
                            d_cv, d_cp, d_ci);
      }
      errors = (got != nnz);
      std::vector<int> gptr = download(d_cp, m + 1);
      std::vector<int> cp32(cp.begin(), cp.end());
      errors += verify(m + 1, gptr.data(), cp32.data());
      if (!errors) {
        std::vector<int> gind = download(d_ci, (size_t)nnz);
        std::vector<float> gval = download(d_cv, (size_t)nnz);
        errors += verify((int)nnz, gind.data(), ci.data());
        std::vector<float> cvf(cv.begin(), cv.end());
        errors += verify((int)nnz, gval.data(), cvf.data());
      }
      cudaFree(d_cp);
      cudaFree(d_ci);
      cudaFree(d_cv);
      cudaFree(d_tp);
      cudaFree(d_ti);
      cudaFree(d_tv);
    } else if (algo == "tc") {
      std::vector<int> perm(m), lp(m + 1), li(g.nnz / 2 + 1);
      orc_tc_build_lower(m, g.ptr.data(), g.ind.data(), perm.data(), lp.data(), li.data());
      long long cpu = orc_tc_lower(m, lp.data(), li.data());
      long long gpu = triangleCount(edge, m, A.d_cscColPtr, A.d_cscRowInd, *context);
      printf("Number of triangles: %lld (CPU %lld)\n", gpu, cpu);
      errors = gpu != cpu;
      printf(errors ? "INCORRECT\n" : "CORRECT\n");
    } else {
      printf("unknown algo %s\n", algo.c_str());
      return 2;
    }
  } catch (const apspie::Error &e) {
    printf("ERROR: %s\n", e.what());
    return 3;
  }
  matrix_delete(&A);
  return errors ? 1 : 0;
}
