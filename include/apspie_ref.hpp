// apspie_ref.hpp -- the reference's host entry points, kept source-compatible
// on top of the C ABI (apspie.h).  A program written against apspie's
// src/*.cuh headers (bfs, sssp, spmspvBfs, spmspvMis, spmspvCsr, mXv,
// spgemm over d_matrix, CompareResults / verify / unverify) compiles against
// this header and runs the sm_100a kernels of libapspie_b200.so instead.
//
// Differences from the reference, all deliberate:
//   * errors throw apspie::Error (the reference prints and exit()s,
//     src/mXv.cuh:12-27) -- the C ABI itself only returns status codes;
//   * sssp runs to convergence; the reference's fixed `depth` iterations with
//     unit weights after the first (src/sssp.cuh:83,91) are not reproduced;
//     unreached vertices are +inf, which its verify() treats like -1
//     (src/util.cuh:230);
//   * spmspvMis takes any order-preserving 32-bit priority: float priorities
//     in (0, 1] (the reference's cuRAND draws) are used through their bit
//     patterns, uint32 priorities (mt19937) directly;
//   * spgemm ignores partSize / partNum (no 2-D tiling is needed);
//   * csr2csc takes the context as a last argument (the reference creates
//     a cuSPARSE handle inside; here the context carries the stream).
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "apspie.h"

namespace apspie {

struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string &msg) : std::runtime_error(msg), status(st) {}
};

inline void check(int st, apspie_ctx ctx, const char *what) {
  if (st != APSPIE_OK)
    throw Error(st, std::string(what) + ": " + (ctx ? apspie_last_error(ctx) : "") + " (" +
                        apspie_status_string(st) + ")");
}

}  // namespace apspie

// mgpu::CudaContext stand-in (the reference creates one per driver with
// mgpu::CreateCudaDevice(0), test/bfs/main.cu:27).
namespace mgpu {
class CudaContext {
 public:
  explicit CudaContext(int device = 0, cudaStream_t stream = nullptr) : stream_(stream) {
    apspie::check(apspie_ctx_create(device, stream, &h_), nullptr, "apspie_ctx_create");
  }
  ~CudaContext() { apspie_ctx_destroy(h_); }
  CudaContext(const CudaContext &) = delete;
  CudaContext &operator=(const CudaContext &) = delete;
  apspie_ctx handle() const { return h_; }
  cudaStream_t Stream() const { return stream_; }
  // The graph passed to bfs() is symmetric (the reference's -undirected
  // flag): the pull direction may then read the same arrays.
  void SetUndirected(bool u) { undirected_ = u; }
  bool Undirected() const { return undirected_; }

 private:
  apspie_ctx h_ = nullptr;
  cudaStream_t stream_ = nullptr;
  bool undirected_ = false;
};
typedef std::shared_ptr<CudaContext> ContextPtr;
inline ContextPtr CreateCudaDevice(int device) { return std::make_shared<CudaContext>(device); }
}  // namespace mgpu

// d_scratch (src/scratch.hpp:5-31): the context owns the workspace, so the
// scratch object carries nothing; allocScratch (src/util.cuh:646) is kept so
// call sites compile.
typedef struct scratch {
  int edge = 0, m = 0;
} d_scratch;
inline void allocScratch(d_scratch **d, const int edge, const int m) {
  *d = new d_scratch;
  (*d)->edge = edge;
  (*d)->m = m;
}

// d_matrix (src/matrix.hpp:6-37), CSR part.  As in the reference, the
// "csc" names hold the CSR of the stored rows.
typedef struct matrix {
  int *d_cscColPtr = nullptr;
  int *d_cscRowInd = nullptr;
  float *d_cscVal = nullptr;
  int *h_cscColPtr = nullptr;
  int *h_cscRowInd = nullptr;
  float *h_cscVal = nullptr;
  int m = 0, n = 0, nnz = 0;
  bool owned_by_library = false;
} d_matrix;

inline void matrix_new(d_matrix *A, int m, int n) {
  A->m = m;
  A->n = n;
  A->nnz = 0;
  A->h_cscColPtr = (int *)calloc((size_t)m + 1, sizeof(int));
  if (!A->h_cscColPtr || cudaMalloc(&A->d_cscColPtr, sizeof(int) * ((size_t)m + 1)) != cudaSuccess)
    throw apspie::Error(APSPIE_ERR_OOM, "matrix_new");
}

// buildMatrix (src/matrix.cpp:56-111): host counting sort of a COO list by
// row (file order kept inside a row), then upload.
template <typename typeVal>
void buildMatrix(d_matrix *A, int numEdge, int *h_cooRowInd, int *h_cooColInd,
                 typeVal *h_cooVal) {
  // the COO entries index host arrays here: checked first (the reference
  // trusts them)
  for (int i = 0; i < numEdge; ++i)
    if (h_cooRowInd[i] < 0 || h_cooRowInd[i] >= A->m || h_cooColInd[i] < 0 ||
        h_cooColInd[i] >= A->n)
      throw apspie::Error(APSPIE_ERR_INVALID, "buildMatrix: entry " + std::to_string(i) +
                                                  " outside the matrix");
  A->nnz = numEdge;
  A->h_cscRowInd = (int *)malloc(sizeof(int) * (size_t)(numEdge > 0 ? numEdge : 1));
  A->h_cscVal = (float *)malloc(sizeof(float) * (size_t)(numEdge > 0 ? numEdge : 1));
  if (!A->h_cscRowInd || !A->h_cscVal) throw apspie::Error(APSPIE_ERR_OOM, "buildMatrix");
  std::vector<int> cnt((size_t)A->m + 1, 0);
  for (int i = 0; i < numEdge; ++i) cnt[(size_t)h_cooRowInd[i] + 1]++;
  for (int i = 0; i < A->m; ++i) cnt[(size_t)i + 1] += cnt[(size_t)i];
  for (int i = 0; i <= A->m; ++i) A->h_cscColPtr[i] = cnt[(size_t)i];
  for (int i = 0; i < numEdge; ++i) {
    int d = cnt[(size_t)h_cooRowInd[i]]++;
    A->h_cscRowInd[d] = h_cooColInd[i];
    A->h_cscVal[d] = h_cooVal ? (float)h_cooVal[i] : 1.0f;
  }
  size_t nb = (size_t)(numEdge > 0 ? numEdge : 1);
  if (cudaMalloc(&A->d_cscRowInd, sizeof(int) * nb) != cudaSuccess ||
      cudaMalloc(&A->d_cscVal, sizeof(float) * nb) != cudaSuccess)
    throw apspie::Error(APSPIE_ERR_OOM, "buildMatrix");
  if (cudaMemcpy(A->d_cscColPtr, A->h_cscColPtr, sizeof(int) * ((size_t)A->m + 1),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(A->d_cscRowInd, A->h_cscRowInd, sizeof(int) * nb, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(A->d_cscVal, A->h_cscVal, sizeof(float) * nb, cudaMemcpyHostToDevice) !=
          cudaSuccess)
    throw apspie::Error(APSPIE_ERR_CUDA, "buildMatrix: upload");
}

inline void matrix_delete(d_matrix *A) {
  if (A->owned_by_library) {
    apspie_csr c{A->m, A->n, A->nnz, A->d_cscColPtr, A->d_cscRowInd, A->d_cscVal};
    apspie_csr_free(nullptr, &c);
  } else {
    cudaFree(A->d_cscColPtr);
    cudaFree(A->d_cscRowInd);
    cudaFree(A->d_cscVal);
  }
  free(A->h_cscColPtr);
  free(A->h_cscRowInd);
  free(A->h_cscVal);
  *A = d_matrix();
}

// ---------------------------------------------------------------- BFS ---
// bfs<T>() (src/bfs.cuh:33): depth = iteration count as in the reference
// (levels 1..depth-1 are assigned); d_cscValA is unused (BFS values are 1).
template <typename T>
void bfs(const int vertex, const int edge, const int m, const T *d_cscValA,
         const int *d_cscColPtrA, const int *d_cscRowIndA, int *d_bfsResult, const int depth,
         mgpu::CudaContext &context) {
  (void)d_cscValA;
  const int *tp = context.Undirected() ? d_cscColPtrA : nullptr;
  const int *ti = context.Undirected() ? d_cscRowIndA : nullptr;
  apspie::check(apspie_bfs(context.handle(), vertex, edge, m, d_cscColPtrA, d_cscRowIndA, tp, ti,
                           d_bfsResult, depth),
                context.handle(), "bfs");
}

// spmspvBfs (src/spmspvBfs.cuh:96): the keys-only variant, same result.
inline void spmspvBfs(const int vertex, const int edge, const int m, const int *h_csrRowPtr,
                      const int *d_csrRowPtr, const int *d_csrColInd, int *d_bfsResult,
                      const int depth, mgpu::CudaContext &context) {
  (void)h_csrRowPtr;
  bfs<int>(vertex, edge, m, nullptr, d_csrRowPtr, d_csrColInd, d_bfsResult, depth, context);
}

// ---------------------------------------------------------------- SSSP ---
template <typename Value>
void sssp(const int vertex, const int edge, const int m, const Value *d_csrValA,
          const int *d_csrRowPtrA, const int *d_csrColIndA, Value *d_ssspResult, const int depth,
          mgpu::CudaContext &context) {
  (void)depth;
  static_assert(std::is_same<Value, float>::value || std::is_same<Value, uint32_t>::value,
                "sssp: float or uint32 weights");
  int st;
  if (std::is_same<Value, float>::value)
    st = apspie_sssp_f32(context.handle(), vertex, edge, m, d_csrRowPtrA, d_csrColIndA,
                         (const float *)d_csrValA, (float *)d_ssspResult, 0);
  else
    st = apspie_sssp_u32(context.handle(), vertex, edge, m, d_csrRowPtrA, d_csrColIndA,
                         (const uint32_t *)d_csrValA, (uint32_t *)d_ssspResult, 0);
  apspie::check(st, context.handle(), "sssp");
}

// spmspvSssp<V>() (src/spmspvSssp.cuh:92): one min-plus SpMSpV, dense in/out.
template <typename Value>
void spmspvSssp(const Value *d_randVec, const int edge, const int m, const Value *d_csrVal,
                const int *d_csrRowPtr, const int *d_csrColInd, Value *d_misResult,
                mgpu::CudaContext &context) {
  static_assert(std::is_same<Value, float>::value, "spmspvSssp: float values");
  apspie::check(apspie_mxv_dense(context.handle(), APSPIE_MIN_PLUS, m, edge, d_csrRowPtr,
                                 d_csrColInd, (const float *)d_csrVal, (const float *)d_randVec,
                                 (float *)d_misResult, nullptr),
                context.handle(), "spmspvSssp");
}

// ----------------------------------------------------------------- MIS ---
template <typename typeVal>
void spmspvMis(const int edge, const int m, const int *h_csrRowPtr, const int *d_csrRowPtr,
               const int *d_csrColInd, const typeVal *d_randVec, int *d_misResult,
               const float delta, mgpu::CudaContext &context) {
  static_assert(sizeof(typeVal) == 4, "spmspvMis: 32-bit priorities");
  (void)h_csrRowPtr;
  apspie::check(apspie_mis(context.handle(), edge, m, d_csrRowPtr, d_csrColInd,
                           (const uint32_t *)d_randVec, d_misResult, delta),
                context.handle(), "spmspvMis");
}

// spmspvCsr (src/spmspvMis.cuh:81): neighbour flags of a vertex set.
template <typename T>
void spmspvCsr(const T *d_inputVector, const int edge, const int m, const int *d_csrRowPtr,
               const int *d_csrColInd, T *d_spmspvResult, mgpu::CudaContext &context) {
  static_assert(sizeof(T) == 4, "spmspvCsr: int flags");
  apspie::check(apspie_neighbor_flags(context.handle(), edge, m, d_csrRowPtr, d_csrColInd,
                                      (const int32_t *)d_inputVector, (int32_t *)d_spmspvResult),
                context.handle(), "spmspvCsr");
}

// ----------------------------------------------------------------- mXv ---
// Dense form (src/mXv.cuh:111): returns the number of products (`total`).
template <typename T>
int mXv(const T *d_randVec, const int edge, const int m, const T *d_cscVal,
        const int *d_cscColPtr, const int *d_cscRowInd, T *d_mmResult, d_scratch *d,
        mgpu::CudaContext &context) {
  static_assert(std::is_same<T, float>::value, "mXv: float values (the kernels compute in float)");
  (void)d;
  int64_t total = 0;
  apspie::check(apspie_mxv_dense(context.handle(), APSPIE_PLUS_TIMES, m, edge, d_cscColPtr,
                                 d_cscRowInd, (const float *)d_cscVal, (const float *)d_randVec,
                                 (float *)d_mmResult, &total),
                context.handle(), "mXv");
  return (int)total;
}

// Sparse form (src/mXv.cuh:250): nnz in = nnz(x), out = nnz(y).
template <typename T>
void mXv(const int *d_randVecInd, const T *d_randVecVal, const int edge, const int m, int &nnz,
         const T *d_cscVal, const int *d_cscColPtr, const int *d_cscRowInd, int *d_resultInd,
         T *d_resultVal, d_scratch *d, mgpu::CudaContext &context) {
  static_assert(std::is_same<T, float>::value, "mXv: float values (the kernels compute in float)");
  (void)d;
  int out = 0;
  apspie::check(apspie_spmspv(context.handle(), APSPIE_PLUS_TIMES, m, edge, d_cscColPtr,
                              d_cscRowInd, (const float *)d_cscVal, nnz, d_randVecInd,
                              (const float *)d_randVecVal, d_resultInd, (float *)d_resultVal,
                              &out, nullptr),
                context.handle(), "mXv");
  nnz = out;
}

// Dense SpMV spmv<T>() (src/bfs.cuh:11-14, mgpu::SpmvCsrBinary): y = A x over
// every row of the CSR (plus-times; the sum is taken in double).
template <typename T>
void spmv(const T *d_inputVector, const int edge, const int m, const T *d_csrValA,
          const int *d_csrRowPtrA, const int *d_csrColIndA, T *d_spmvResult,
          mgpu::CudaContext &context) {
  static_assert(std::is_same<T, float>::value, "spmv: float values");
  apspie::check(apspie_spmv(context.handle(), APSPIE_PLUS_TIMES, m, edge, d_csrRowPtrA,
                            d_csrColIndA, (const float *)d_csrValA, (const float *)d_inputVector,
                            (float *)d_spmvResult),
                context.handle(), "spmv");
}

// csr2csc<T>() (src/util.cuh:473-488): transpose of a square CSR, values
// carried along, row ids ascending within each column.
template <typename typeVal>
void csr2csc(const int m, const int edge, const typeVal *d_csrValA, const int *d_csrRowPtrA,
             const int *d_csrColIndA, typeVal *d_cscValA, int *d_cscRowIndA, int *d_cscColPtrA,
             mgpu::CudaContext &context) {
  static_assert(std::is_same<typeVal, float>::value, "csr2csc: float values");
  apspie::check(apspie_csr_transpose(context.handle(), m, m, edge, d_csrRowPtrA, d_csrColIndA,
                                     (const float *)d_csrValA, d_cscColPtrA, d_cscRowIndA,
                                     (float *)d_cscValA),
                context.handle(), "csr2csc");
}

// -------------------------------------------------------------- SpGEMM ---
// spgemm(d_matrix *C, A, B, partSize, partNum, ctx) (src/spgemm.cuh:132).
// C's device arrays are allocated by the library (release: matrix_delete).
inline void spgemm(d_matrix *C, d_matrix *A, d_matrix *B, const int partSize, const int partNum,
                   mgpu::CudaContext &context) {
  (void)partSize;
  (void)partNum;
  apspie_csr a{A->m, A->n, A->nnz, A->d_cscColPtr, A->d_cscRowInd, A->d_cscVal};
  apspie_csr b{B->m, B->n, B->nnz, B->d_cscColPtr, B->d_cscRowInd, B->d_cscVal};
  apspie_csr c{};
  apspie::check(apspie_spgemm(context.handle(), &a, &b, &c), context.handle(), "spgemm");
  C->m = c.m;
  C->n = c.n;
  C->nnz = (int)c.nnz;
  C->d_cscColPtr = c.d_ptr;
  C->d_cscRowInd = c.d_ind;
  C->d_cscVal = c.d_val;
  C->owned_by_library = true;
}

// spgemm<T>() (src/tc.cuh:63-165): C = A * B on the arrays as given -- the
// reference hands its "csc" arrays to cusparseXcsrgemmNnz / cusparseScsrgemm,
// which read them as CSR, so the TC driver's call spgemm(C, B) forms U * L
// (test/tc/main.cu:241).  C's arrays are allocated here with cudaMalloc, as
// the reference allocates them (src/tc.cuh:73,120-121); the caller frees them
// with cudaFree.  `edge` is the reference's nnz argument for both inputs
// (the TC driver passes the whole graph's edge count for its half
// matrices); here nnz(A) and nnz(B) are read from the offsets.  The call
// runs on a context of its own, as the reference creates its own cuSPARSE
// handle.  Returns nnz(C).
template <typename T>
int spgemm(const int edge, const int m, const T *d_cscValA, const int *d_cscColPtrA,
           const int *d_cscRowIndA, const T *d_cscValB, const int *d_cscColPtrB,
           const int *d_cscRowIndB, T *&d_cscValC, int *&d_cscColPtrC, int *&d_cscRowIndC) {
  static_assert(std::is_same<T, float>::value, "spgemm<T>: float values, as cusparseScsrgemm");
  (void)edge;
  int dev = 0, na = 0, nb = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaMemcpy(&na, d_cscColPtrA + m, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&nb, d_cscColPtrB + m, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    throw apspie::Error(APSPIE_ERR_CUDA, "spgemm: reading the offsets");
  mgpu::CudaContext ctx(dev);
  apspie_csr a{m, m, na, const_cast<int *>(d_cscColPtrA), const_cast<int *>(d_cscRowIndA),
               const_cast<float *>((const float *)d_cscValA)};
  apspie_csr b{m, m, nb, const_cast<int *>(d_cscColPtrB), const_cast<int *>(d_cscRowIndB),
               const_cast<float *>((const float *)d_cscValB)};
  apspie_csr c{};
  apspie::check(apspie_spgemm(ctx.handle(), &a, &b, &c), ctx.handle(), "spgemm");
  d_cscValC = (T *)c.d_val;
  d_cscColPtrC = c.d_ptr;
  d_cscRowIndC = c.d_ind;
  return (int)c.nnz;
}

// mXm<T>() (src/tc.cuh:315-375): C(:, i) = A * B(:, i) for every column i of
// B (the reference runs one sparse mXv per column), i.e. C = A * B on the
// CSC arrays.  Read as CSR arrays these hold the transposes, so C's arrays
// are the CSR product of B's arrays and A's (apspie_spgemm(B, A)); each
// column comes out with its rows ascending, as mXv's ReduceByKey leaves
// them.  The reference allocates C inside, through its by-value pointer
// parameters, and so never returns it (src/tc.cuh:318-324); here C is
// written into the caller's arrays: d_cscColPtrC m + 1 offsets, and
// d_cscRowIndC / d_cscValC nnz(C) entries, at most the 16 * edge the
// reference sizes them for (a larger product throws APSPIE_ERR_TOO_LARGE
// before anything is written but the offsets).  Returns nnz(C).
template <typename T>
int mXm(const int edge, const int m, const T *d_cscValA, const int *d_cscColPtrA,
        const int *d_cscRowIndA, const T *d_cscValB, const int *h_cscColPtrB,
        const int *d_cscColPtrB, const int *d_cscRowIndB, T *d_cscValC, int *d_cscColPtrC,
        int *d_cscRowIndC, mgpu::CudaContext &context) {
  static_assert(std::is_same<T, float>::value, "mXm<T>: float values");
  int na = 0;
  if (cudaMemcpy(&na, d_cscColPtrA + m, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    throw apspie::Error(APSPIE_ERR_CUDA, "mXm: reading the offsets");
  apspie_csr a{m, m, na, const_cast<int *>(d_cscColPtrA), const_cast<int *>(d_cscRowIndA),
               const_cast<float *>((const float *)d_cscValA)};
  apspie_csr b{m, m, h_cscColPtrB[m], const_cast<int *>(d_cscColPtrB),
               const_cast<int *>(d_cscRowIndB), const_cast<float *>((const float *)d_cscValB)};
  int64_t nnz = 0;
  apspie::check(apspie_spgemm_symbolic(context.handle(), &b, &a, d_cscColPtrC, &nnz),
                context.handle(), "mXm");
  if (nnz > 16ll * edge)
    throw apspie::Error(APSPIE_ERR_TOO_LARGE, "mXm: nnz(C) exceeds 16 * edge");
  apspie::check(apspie_spgemm_numeric(context.handle(), &b, &a, d_cscColPtrC, d_cscRowIndC,
                                      (float *)d_cscValC),
                context.handle(), "mXm");
  apspie::check(apspie_ctx_sync(context.handle()), context.handle(), "mXm");
  return (int)nnz;
}

// Triangle count of a symmetric graph (the computation of test/tc/main.cu).
inline long long triangleCount(const int edge, const int m, const int *d_ptr, const int *d_ind,
                               mgpu::CudaContext &context) {
  int *perm = nullptr, *lp = nullptr, *li = nullptr;
  int64_t lnnz = 0, count = 0;
  int st = APSPIE_OK;
  if (cudaMalloc(&perm, sizeof(int) * (size_t)m) != cudaSuccess ||
      cudaMalloc(&lp, sizeof(int) * ((size_t)m + 1)) != cudaSuccess ||
      cudaMalloc(&li, sizeof(int) * (size_t)(edge / 2 + 1)) != cudaSuccess) {
    cudaGetLastError();
    st = APSPIE_ERR_OOM;
  }
  if (st == APSPIE_OK)
    st = apspie_tc_prepare(context.handle(), edge, m, d_ptr, d_ind, perm, lp, li, &lnnz);
  if (st == APSPIE_OK) st = apspie_tc(context.handle(), m, lnnz, lp, li, &count);
  cudaFree(perm);
  cudaFree(lp);
  cudaFree(li);
  apspie::check(st, context.handle(), "triangleCount");
  return count;
}

// ---------------------------------------------------- result checking ---
// CompareResults (src/util.cuh:187-257): exact for integers; for float, -1 and
// >= 1e38 both mean "unreached" and values within 10 % relative count as
// equal.  Returns the number of mismatches and prints CORRECT when none.
template <typename T>
int CompareResults(const T *computed, const T *reference, const int len,
                   const bool verbose = true) {
  int errors = 0;
  for (int i = 0; i < len; ++i) {
    bool bad;
    if (std::is_floating_point<T>::value) {
      double c = (double)computed[i], r = (double)reference[i];
      bool cu = (c == -1.0 || c > 1e38 || std::isinf(c)), ru = (r == -1.0 || r > 1e38 || std::isinf(r));
      bad = (cu != ru) || (!cu && std::fabs(c - r) > 0.1 * std::fabs(c));
    } else {
      bad = computed[i] != reference[i];
    }
    if (bad && errors == 0 && verbose)
      std::cout << "\nINCORRECT: [" << i << "]: " << computed[i] << " != " << reference[i];
    errors += bad;
  }
  std::cout << "\n" << (errors ? "" : "CORRECT\n");
  return errors;
}

template <typename value>
int verify(const int m, const value *h_result, const value *h_resultCPU) {
  std::cout << "Label Validity: ";
  int e = CompareResults(h_result, h_resultCPU, m, true);
  if (e > 0) std::cout << e << " errors occurred.\n";
  return e;
}

// unverify (src/util.cuh:272-316): computed + reference must be 1 everywhere
// (the MIS check: neighbour flag + membership).
inline int unverify(const int m, const int *h_result, const int *h_resultCPU) {
  std::cout << "Label Validity: ";
  int errors = 0;
  for (int i = 0; i < m; ++i) errors += (h_result[i] + h_resultCPU[i] != 1);
  std::cout << "\n" << (errors ? "" : "CORRECT\n");
  if (errors) std::cout << errors << " errors occurred.\n";
  return errors;
}
