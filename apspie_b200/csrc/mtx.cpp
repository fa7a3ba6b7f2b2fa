// mtx.cpp -- Matrix Market ingest with the reference's orientation.
//
// readEdge / readMtx (src/util.cuh:355-430): '%' lines are skipped, then
// "m n nnz", then one entry per line.  The FIRST index of a line is stored as
// the column and the SECOND as the row, both made 0-based; a line is weighted
// when the first entry carries a third token.  The CSR built from it
// (buildMatrix, src/matrix.cpp:56-111) keeps the file order inside each row.
// With undirected != 0 the edges are symmetrised as makeSymmetric does
// (src/util.cuh:573-643): every non-loop entry gets its mirror, entries are
// sorted by (row, col), repeats are dropped and self-loops are kept.  Unlike
// the reference, values stay aligned with their entries after the compaction.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "apspie.h"

namespace {

struct Entry {
  int row, col;
  float val;
};

int emit_csr(int m, const std::vector<Entry> &e, int **h_ptr, int **h_ind, float **h_val) {
  int *ptr = (int *)malloc(sizeof(int) * ((size_t)m + 1));
  int *ind = (int *)malloc(sizeof(int) * (e.empty() ? 1 : e.size()));
  float *val = h_val ? (float *)malloc(sizeof(float) * (e.empty() ? 1 : e.size())) : nullptr;
  if (!ptr || !ind || (h_val && !val)) {
    free(ptr);
    free(ind);
    free(val);
    return APSPIE_ERR_OOM;
  }
  std::vector<int> cnt((size_t)m + 1, 0);
  for (auto &x : e) cnt[(size_t)x.row + 1]++;
  for (int i = 0; i < m; ++i) cnt[(size_t)i + 1] += cnt[(size_t)i];
  for (int i = 0; i <= m; ++i) ptr[i] = cnt[(size_t)i];
  for (auto &x : e) {  // stable counting sort by row
    int d = cnt[(size_t)x.row]++;
    ind[d] = x.col;
    if (val) val[d] = x.val;
  }
  *h_ptr = ptr;
  *h_ind = ind;
  if (h_val) *h_val = val;
  return APSPIE_OK;
}

// Parses an opened file (apspie_read_mtx_host opens and closes it).
int read_mtx(FILE *f, int undirected, int *m_out, int64_t *nnz_out, int **h_ptr, int **h_ind,
             float **h_val, int *weighted_out) {
  char line[4096];
  long long m = -1, n = -1, nz = -1;
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '%') continue;
    if (sscanf(line, "%lld %lld %lld", &m, &n, &nz) == 3) break;
  }
  if (m < 0 || nz < 0 || m >= INT32_MAX || nz >= INT32_MAX) return APSPIE_ERR_INVALID;
  std::vector<Entry> e;
  // the header's count is only a hint: a short file must not cost the
  // memory of a long one
  e.reserve(std::min<size_t>((size_t)nz * (undirected ? 2 : 1), size_t(1) << 24));
  int weighted = -1;
  for (long long k = 0; k < nz; ++k) {
    if (!fgets(line, sizeof(line), f)) break;  // fewer entries than promised
    long long a, b;
    double w = 1.0;
    int got = sscanf(line, "%lld %lld %lf", &a, &b, &w);
    if (got < 2) {
      --k;
      continue;
    }
    if (weighted < 0) weighted = (got == 3);
    if (!weighted) w = 1.0;
    if (a < 1 || b < 1 || a > m || b > m) return APSPIE_ERR_INVALID;
    e.push_back(Entry{(int)(b - 1), (int)(a - 1), (float)w});
  }
  if (undirected) {
    size_t n0 = e.size();
    for (size_t i = 0; i < n0; ++i)
      if (e[i].row != e[i].col) e.push_back(Entry{e[i].col, e[i].row, e[i].val});
    std::stable_sort(e.begin(), e.end(), [](const Entry &x, const Entry &y) {
      return x.row != y.row ? x.row < y.row : x.col < y.col;
    });
    size_t w = 0;
    for (size_t i = 0; i < e.size(); ++i)
      if (w == 0 || e[i].row != e[w - 1].row || e[i].col != e[w - 1].col) e[w++] = e[i];
    e.resize(w);
  }
  if (e.size() >= (size_t)INT32_MAX) return APSPIE_ERR_OVERFLOW;  // int32 row offsets
  *m_out = (int)m;
  *nnz_out = (int64_t)e.size();
  if (weighted_out) *weighted_out = weighted > 0;
  return emit_csr((int)m, e, h_ptr, h_ind, h_val);
}

}  // namespace

extern "C" {

int apspie_read_mtx_host(const char *path, int undirected, int *m_out, int64_t *nnz_out,
                         int **h_ptr, int **h_ind, float **h_val, int *weighted_out) {
  if (!path || !m_out || !nnz_out || !h_ptr || !h_ind) return APSPIE_ERR_INVALID;
  FILE *f = fopen(path, "r");
  if (!f) return APSPIE_ERR_INVALID;
  int st;
  try {  // no C++ exception leaves the C ABI
    st = read_mtx(f, undirected, m_out, nnz_out, h_ptr, h_ind, h_val, weighted_out);
  } catch (const std::bad_alloc &) {
    st = APSPIE_ERR_OOM;
  }
  fclose(f);
  return st;
}

}  // extern "C"
