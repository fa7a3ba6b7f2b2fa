/*
 * oracle.h -- CPU restatement of apspie's SpMSpV / hash-SpGEMM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may
 * load it.  The product (apspie_b200) never links or calls it.
 *
 * Every function names the reference file:line whose behaviour it restates
 * (paths are relative to the apspie source tree).  Parity is pinned two ways:
 *   - against the reference's own CPU BFS / SSSP / MT19937, compiled from the
 *     reference sources into oracle/_ref/ by oracle/Makefile, on every
 *     fixture graph and on seeded synthetic graphs (tests/test_oracle_pin.py);
 *   - against golden vectors generated from those compiled reference routines
 *     and committed under tests/golden/ (tests/golden/make_golden.py).
 * MIS, TC, SpGEMM and SpMSpV have no CPU implementation in the reference;
 * their restatements follow the GPU code's semantics and are pinned by the
 * structural rules the reference's tests apply (MIS validity, SpGEMM
 * structure) -- see the comment on each function.
 */
#ifndef APSPIE_ORACLE_H
#define APSPIE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Queue BFS.  src/testBfs.cpp:7-72 (SimpleReferenceBfs) and :75-90 (bfsCPU).
 * depth[v] = hops from src, -1 if unreached, depth[src] = 0.  Expansion stops
 * once a vertex whose neighbours would get depth > stop is dequeued.
 * Returns the search depth (deepest level + 1), as the reference does. */
int orc_bfs(int m, const int *rowptr, const int *colind, int src, int stop,
            int *depth);

/* Label-correcting priority-queue SSSP in float arithmetic,
 * src/testSssp.cpp:33-115 (SimpleReferenceSssp).  dist[v] = -1 if unreached.
 * Each relaxation computes fl32(dist[u] + w) exactly as the reference does,
 * so the result is the unique float fixpoint of min over in-edges. */
void orc_sssp_f32(int m, const int *rowptr, const int *colind, const float *w,
                  int src, float *dist);

/* Same algorithm with double accumulation (the FP64 oracle for the 1e-6
 * tolerance on float SSSP).  dist[v] = +inf if unreached. */
void orc_sssp_f64(int m, const int *rowptr, const int *colind, const float *w,
                  int src, double *dist);

/* Same algorithm on uint32 weights; dist[v] = UINT32_MAX if unreached.
 * Sums are formed in 64 bits and saturate at UINT32_MAX - 1. */
void orc_sssp_u32(int m, const int *rowptr, const int *colind,
                  const uint32_t *w, int src, uint32_t *dist);

/* Maximal independent set with fixed priorities, restating the round
 * structure of src/spmspvMis.cuh:54-78 (buildVector / updateMis /
 * updateNeighbor) and :232-318 (round loop).  With fixed priorities a vertex
 * joins exactly when it beats every undecided neighbour, so the final set is
 * the greedy MIS in descending key order; key(v) = (prio[v] << 32) | v (ties
 * in priority go to the larger vertex id).  Self-loops are ignored.
 * mis[v] = 1 (in set) or 0 (adjacent to the set). */
void orc_mis(int m, const int *rowptr, const int *colind, const uint32_t *prio,
             int *mis);

/* Neighbour flags of a vertex set: out[v] = 1 if v is adjacent to some u with
 * in[u] != 0, else 0.  src/spmspvMis.cuh:81-147 (spmspvCsr), used by the MIS
 * check in test/mis/main.cu:217-221. */
void orc_neighbor_flags(int m, const int *rowptr, const int *colind,
                        const int *in, int *out);

/* MIS validity rule of test/mis/main.cu:217-221 with src/util.cuh:272-306
 * (uncompareResults): every vertex must satisfy flag(v) + mis(v) == 1, where
 * flag = orc_neighbor_flags(mis).  Returns the number of violating vertices. */
int orc_mis_check(int m, const int *rowptr, const int *colind, const int *mis);

/* Degree-ordered strict-lower triangle for triangle counting.
 * test/tc/main.cu:40-55 (buildLower) after relabelling vertices by ascending
 * (degree, id).  perm[v] = new id of v.  Lptr has m+1 entries; Lind must hold
 * nnz/2 entries (self-loops are dropped).  Rows are sorted ascending.
 * Returns nnz(L). */
int orc_tc_build_lower(int m, const int *rowptr, const int *colind, int *perm,
                       int *Lptr, int *Lind);

/* Triangle count sum_{(i,j) in L} |L(i,:) n L(j,:)| in int64, the value that
 * test/tc/main.cu:243-261 (cuSPARSE U*L then ewiseMultTc, src/tc.cuh:169-199)
 * computes in float. */
int64_t orc_tc_lower(int m, const int *Lptr, const int *Lind);

/* Gustavson SpGEMM C = A*B, symbolic part: Cptr[i+1]-Cptr[i] = number of
 * distinct columns j with some A(i,k)B(k,j) (explicit zeros kept, as the
 * reference hash insert keeps any touched key, src/spgemmKernel.cuh:179-208).
 * Cptr has m+1 entries.  Returns nnz(C). */
int64_t orc_spgemm_symbolic(int m, int n, const int *Aptr, const int *Aind,
                            const int *Bptr, const int *Bind, int64_t *Cptr);

/* Numeric part: columns ascending per row (src/spgemmKernel.cuh:698-715),
 * values accumulated in double. */
void orc_spgemm_numeric(int m, int n, const int *Aptr, const int *Aind,
                        const float *Aval, const int *Bptr, const int *Bind,
                        const float *Bval, const int64_t *Cptr, int *Cind,
                        double *Cval);

/* Semirings for orc_spmspv. */
enum {
  ORC_PLUS_TIMES = 0, /* mXv:        y = sum  A(r,j)*x[j]  (src/mXv.cuh:106,201) */
  ORC_MIN_PLUS = 1,   /* spmspvSssp: y = min  A(r,j)+x[j]  (src/spmspvSssp.cuh:87,232) */
  ORC_MAX_TIMES = 2,  /* spmspvMis:  y = max  A(r,j)*x[j]  (src/spmspvMis.cuh:289) */
  ORC_OR_AND = 3      /* Boolean:    y = 1 if any A(r,j)x[j] structurally present */
};

/* Sparse x times A given as column lists (ptr/ind/val = CSC of A, i.e. the
 * out-adjacency of each frontier vertex), src/mXv.cuh:250-389.  Output is
 * sorted by row index with one entry per touched row (structural).  val may
 * be NULL (all ones).  PLUS_TIMES accumulates in double; MIN_PLUS and
 * MAX_TIMES form each term in float as the reference does.
 * Returns nnz(y). */
int orc_spmspv(int semiring, int m, const int *ptr, const int *ind,
               const float *val, int xnnz, const int *xind, const float *xval,
               int *yind, double *yval);

/* MT19937 (Matsumoto & Nishimura 2002), as in src/mt19937ar.cpp:57-150,
 * with explicit state.  orc_mt_fill writes genrand_int32() n times after
 * init_genrand(seed). */
void orc_mt_fill(uint32_t seed, int64_t n, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
