/*
 * oracle.c -- CPU restatement of apspie's traversal / SpGEMM semantics.
 * TEST INFRASTRUCTURE ONLY (the checker); see oracle.h for the contract and
 * the reference citations of every function.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- BFS --- */
int orc_bfs(int m, const int *rowptr, const int *colind, int src, int stop,
            int *depth) {
  /* src/testBfs.cpp:17-60: FIFO queue, depth -1 = undiscovered. */
  for (int i = 0; i < m; ++i) depth[i] = -1;
  if (src < 0 || src >= m) return 0;
  int *queue = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  int head = 0, tail = 0, search_depth = 0;
  depth[src] = 0;
  queue[tail++] = src;
  while (head < tail) {
    int u = queue[head++];
    int nd = depth[u] + 1;
    if (nd > stop) break;
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e) {
      int v = colind[e];
      if (depth[v] == -1) {
        depth[v] = nd;
        if (search_depth < nd) search_depth = nd;
        queue[tail++] = v;
      }
    }
  }
  free(queue);
  return search_depth + 1;
}

/* ------------------------------------------------- binary min-heap ------ */
/* Entries are (key, vertex); lazy deletion, as the reference's
 * std::priority_queue with duplicate pushes (src/testSssp.cpp:42-97). */
typedef struct {
  double key;
  int v;
} hent;
typedef struct {
  hent *a;
  size_t n, cap;
} heap;

static void hpush(heap *h, double key, int v) {
  if (h->n == h->cap) {
    h->cap = h->cap ? 2 * h->cap : 1024;
    h->a = (hent *)realloc(h->a, h->cap * sizeof(hent));
  }
  size_t i = h->n++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (h->a[p].key <= key) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i].key = key;
  h->a[i].v = v;
}

static hent hpop(heap *h) {
  hent top = h->a[0];
  hent last = h->a[--h->n];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1;
    if (l >= h->n) break;
    size_t c = (l + 1 < h->n && h->a[l + 1].key < h->a[l].key) ? l + 1 : l;
    if (h->a[c].key >= last.key) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n) h->a[i] = last;
  return top;
}

/* --------------------------------------------------------------- SSSP --- */
void orc_sssp_f32(int m, const int *rowptr, const int *colind, const float *w,
                  int src, float *dist) {
  /* src/testSssp.cpp:49-97.  A vertex is expanded whenever it is popped with
   * a label no worse than its current one; relaxation is fl32(d[u] + w). */
  for (int i = 0; i < m; ++i) dist[i] = -1.0f;
  if (src < 0 || src >= m) return;
  heap h = {0, 0, 0};
  dist[src] = 0.0f;
  hpush(&h, 0.0, src);
  while (h.n) {
    hent t = hpop(&h);
    int u = t.v;
    if ((float)t.key > dist[u]) continue; /* stale entry */
    float du = dist[u];
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e) {
      int v = colind[e];
      volatile float alt = du + w[e]; /* one IEEE single add, no fusion */
      if (dist[v] == -1.0f || alt < dist[v]) {
        dist[v] = alt;
        hpush(&h, (double)alt, v);
      }
    }
  }
  free(h.a);
}

void orc_sssp_f64(int m, const int *rowptr, const int *colind, const float *w,
                  int src, double *dist) {
  for (int i = 0; i < m; ++i) dist[i] = INFINITY;
  if (src < 0 || src >= m) return;
  heap h = {0, 0, 0};
  dist[src] = 0.0;
  hpush(&h, 0.0, src);
  while (h.n) {
    hent t = hpop(&h);
    int u = t.v;
    if (t.key > dist[u]) continue;
    double du = dist[u];
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e) {
      int v = colind[e];
      double alt = du + (double)w[e];
      if (alt < dist[v]) {
        dist[v] = alt;
        hpush(&h, alt, v);
      }
    }
  }
  free(h.a);
}

void orc_sssp_u32(int m, const int *rowptr, const int *colind,
                  const uint32_t *w, int src, uint32_t *dist) {
  for (int i = 0; i < m; ++i) dist[i] = UINT32_MAX;
  if (src < 0 || src >= m) return;
  heap h = {0, 0, 0};
  dist[src] = 0;
  hpush(&h, 0.0, src);
  while (h.n) {
    hent t = hpop(&h);
    int u = t.v;
    if ((uint32_t)t.key > dist[u]) continue;
    uint64_t du = dist[u];
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e) {
      int v = colind[e];
      uint64_t alt = du + w[e];
      if (alt > (uint64_t)UINT32_MAX - 1) alt = (uint64_t)UINT32_MAX - 1;
      if (alt < dist[v]) {
        dist[v] = (uint32_t)alt;
        hpush(&h, (double)alt, v);
      }
    }
  }
  free(h.a);
}

/* ---------------------------------------------------------------- MIS --- */
static const uint32_t *g_prio; /* qsort has no context argument */
static int cmp_key_desc(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  uint64_t kx = ((uint64_t)g_prio[x] << 32) | (uint32_t)x;
  uint64_t ky = ((uint64_t)g_prio[y] << 32) | (uint32_t)y;
  return kx < ky ? 1 : (kx > ky ? -1 : 0);
}

void orc_mis(int m, const int *rowptr, const int *colind, const uint32_t *prio,
             int *mis) {
  /* Round r of src/spmspvMis.cuh:232-318 admits every undecided vertex that
   * beats all undecided neighbours (updateMis :64) and removes the
   * neighbours of the admitted ones (updateNeighbor :71).  Processing the
   * vertices once in descending key order admits exactly the same set. */
  int *order = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  for (int i = 0; i < m; ++i) {
    order[i] = i;
    mis[i] = -1;
  }
  g_prio = prio;
  qsort(order, (size_t)m, sizeof(int), cmp_key_desc);
  for (int t = 0; t < m; ++t) {
    int v = order[t];
    if (mis[v] != -1) continue;
    mis[v] = 1;
    for (int e = rowptr[v]; e < rowptr[v + 1]; ++e) {
      int u = colind[e];
      if (u != v && mis[u] == -1) mis[u] = 0;
    }
  }
  free(order);
}

void orc_neighbor_flags(int m, const int *rowptr, const int *colind,
                        const int *in, int *out) {
  for (int i = 0; i < m; ++i) out[i] = 0;
  for (int u = 0; u < m; ++u) {
    if (!in[u]) continue;
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e) out[colind[e]] = 1;
  }
}

int orc_mis_check(int m, const int *rowptr, const int *colind, const int *mis) {
  int *in = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  int *fl = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  for (int i = 0; i < m; ++i) in[i] = mis[i] == 1;
  orc_neighbor_flags(m, rowptr, colind, in, fl);
  int errors = 0;
  for (int i = 0; i < m; ++i)
    if (fl[i] + (mis[i] == 1 ? 1 : (mis[i] == 0 ? 0 : 7)) != 1) ++errors;
  free(in);
  free(fl);
  return errors;
}

/* ----------------------------------------------------------------- TC --- */
static const int *g_deg;
static int cmp_deg_asc(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  if (g_deg[x] != g_deg[y]) return g_deg[x] < g_deg[y] ? -1 : 1;
  return x < y ? -1 : (x > y);
}
static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return x < y ? -1 : (x > y);
}

int orc_tc_build_lower(int m, const int *rowptr, const int *colind, int *perm,
                       int *Lptr, int *Lind) {
  int *deg = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  int *order = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  for (int v = 0; v < m; ++v) {
    deg[v] = rowptr[v + 1] - rowptr[v];
    order[v] = v;
  }
  g_deg = deg;
  qsort(order, (size_t)m, sizeof(int), cmp_deg_asc);
  for (int r = 0; r < m; ++r) perm[order[r]] = r;
  /* row new(u) of L holds new(v) for every edge u-v with new(v) < new(u) */
  for (int i = 0; i <= m; ++i) Lptr[i] = 0;
  for (int u = 0; u < m; ++u)
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e)
      if (perm[colind[e]] < perm[u]) Lptr[perm[u] + 1]++;
  for (int i = 0; i < m; ++i) Lptr[i + 1] += Lptr[i];
  int *fill = (int *)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
  for (int i = 0; i < m; ++i) fill[i] = Lptr[i];
  for (int u = 0; u < m; ++u)
    for (int e = rowptr[u]; e < rowptr[u + 1]; ++e)
      if (perm[colind[e]] < perm[u]) Lind[fill[perm[u]]++] = perm[colind[e]];
  for (int i = 0; i < m; ++i)
    qsort(Lind + Lptr[i], (size_t)(Lptr[i + 1] - Lptr[i]), sizeof(int), cmp_int);
  free(fill);
  free(order);
  free(deg);
  return Lptr[m];
}

int64_t orc_tc_lower(int m, const int *Lptr, const int *Lind) {
  int64_t count = 0;
  for (int i = 0; i < m; ++i) {
    for (int e = Lptr[i]; e < Lptr[i + 1]; ++e) {
      int j = Lind[e];
      /* sorted-merge intersection, as ewiseMultTc (src/tc.cuh:182-196) */
      int a = Lptr[i], ae = Lptr[i + 1], b = Lptr[j], be = Lptr[j + 1];
      while (a < ae && b < be) {
        int d = Lind[a] - Lind[b];
        if (d == 0) ++count;
        if (d <= 0) ++a;
        if (d >= 0) ++b;
      }
    }
  }
  return count;
}

/* ------------------------------------------------------------- SpGEMM --- */
int64_t orc_spgemm_symbolic(int m, int n, const int *Aptr, const int *Aind,
                            const int *Bptr, const int *Bind, int64_t *Cptr) {
  int *mark = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int j = 0; j < n; ++j) mark[j] = -1;
  Cptr[0] = 0;
  for (int i = 0; i < m; ++i) {
    int64_t c = 0;
    for (int a = Aptr[i]; a < Aptr[i + 1]; ++a) {
      int k = Aind[a];
      for (int b = Bptr[k]; b < Bptr[k + 1]; ++b) {
        int j = Bind[b];
        if (mark[j] != i) {
          mark[j] = i;
          ++c;
        }
      }
    }
    Cptr[i + 1] = Cptr[i] + c;
  }
  free(mark);
  return Cptr[m];
}

void orc_spgemm_numeric(int m, int n, const int *Aptr, const int *Aind,
                        const float *Aval, const int *Bptr, const int *Bind,
                        const float *Bval, const int64_t *Cptr, int *Cind,
                        double *Cval) {
  int *mark = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  double *acc = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  for (int j = 0; j < n; ++j) mark[j] = -1;
  for (int i = 0; i < m; ++i) {
    int64_t c = Cptr[i];
    for (int a = Aptr[i]; a < Aptr[i + 1]; ++a) {
      int k = Aind[a];
      double av = Aval ? (double)Aval[a] : 1.0;
      for (int b = Bptr[k]; b < Bptr[k + 1]; ++b) {
        int j = Bind[b];
        double p = av * (Bval ? (double)Bval[b] : 1.0);
        if (mark[j] != i) {
          mark[j] = i;
          acc[j] = p;
          Cind[c++] = j;
        } else {
          acc[j] += p;
        }
      }
    }
    qsort(Cind + Cptr[i], (size_t)(Cptr[i + 1] - Cptr[i]), sizeof(int), cmp_int);
    for (int64_t t = Cptr[i]; t < Cptr[i + 1]; ++t) Cval[t] = acc[Cind[t]];
  }
  free(acc);
  free(mark);
}

/* ------------------------------------------------------------ SpMSpV --- */
int orc_spmspv(int semiring, int m, const int *ptr, const int *ind,
               const float *val, int xnnz, const int *xind, const float *xval,
               int *yind, double *yval) {
  /* Expand (src/mXv.cuh:329-343), then reduce by row (:373); the result is
   * sorted by row because the reference radix-sorts the keys (:361). */
  unsigned char *touched = (unsigned char *)calloc((size_t)(m > 0 ? m : 1), 1);
  double *acc = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  for (int t = 0; t < xnnz; ++t) {
    int j = xind[t];
    float xv = xval ? xval[t] : 1.0f;
    for (int e = ptr[j]; e < ptr[j + 1]; ++e) {
      int r = ind[e];
      float a = val ? val[e] : 1.0f;
      double term;
      switch (semiring) {
        case ORC_PLUS_TIMES: term = (double)a * (double)xv; break;
        case ORC_MIN_PLUS: { volatile float s = a + xv; term = s; } break;
        case ORC_MAX_TIMES: { volatile float p = a * xv; term = p; } break;
        default: term = 1.0; break;
      }
      if (!touched[r]) {
        touched[r] = 1;
        acc[r] = term;
      } else {
        switch (semiring) {
          case ORC_PLUS_TIMES: acc[r] += term; break;
          case ORC_MIN_PLUS: if (term < acc[r]) acc[r] = term; break;
          case ORC_MAX_TIMES: if (term > acc[r]) acc[r] = term; break;
          default: acc[r] = 1.0; break;
        }
      }
    }
  }
  int n = 0;
  for (int r = 0; r < m; ++r)
    if (touched[r]) {
      yind[n] = r;
      yval[n] = acc[r];
      ++n;
    }
  free(acc);
  free(touched);
  return n;
}

/* ------------------------------------------------------------ MT19937 --- */
void orc_mt_fill(uint32_t seed, int64_t n, uint32_t *out) {
  /* src/mt19937ar.cpp:57-70 (init_genrand) and :112-150 (genrand_int32). */
  enum { NN = 624, MM = 397 };
  uint32_t mt[NN];
  int mti;
  mt[0] = seed;
  for (mti = 1; mti < NN; ++mti)
    mt[mti] = 1812433253u * (mt[mti - 1] ^ (mt[mti - 1] >> 30)) + (uint32_t)mti;
  for (int64_t t = 0; t < n; ++t) {
    if (mti >= NN) {
      for (int k = 0; k < NN; ++k) {
        uint32_t y = (mt[k] & 0x80000000u) | (mt[(k + 1) % NN] & 0x7fffffffu);
        mt[k] = mt[(k + MM) % NN] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
      }
      mti = 0;
    }
    uint32_t y = mt[mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    out[t] = y;
  }
}
