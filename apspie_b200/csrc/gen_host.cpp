// gen_host.cpp -- host builders for the synthetic benchmark graphs.
//
// The reference reads Matrix Market files and symmetrises them with a qsort
// (src/util.cuh:522-643, src/matrix.cpp:56-111); the benchmark graphs here are
// generated instead.  Every random draw is a counter-based splitmix64 hash of
// (seed, sample index), so the same edge multiset comes out on any thread
// count and on the device builder (gen.cu).  Edges are packed as
// (row << 32 | col), radix-sorted with a multi-threaded LSD sort, deduplicated
// and turned into CSR.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <thread>
#include <vector>

#include "apspie.h"
#include "gen_common.h"

namespace {

int num_threads() {
  unsigned n = std::thread::hardware_concurrency();
  if (n == 0) n = 1;
  if (n > 64) n = 64;
  return (int)n;
}

// f(b, e, t) over [0, n) in num_threads() chunks, chunk t = [t * per,
// (t + 1) * per).  A chunk whose thread cannot be started runs on the
// calling thread instead, so the chunks are the same and nothing is thrown
// once threads are running (a joinable std::thread must not be destroyed).
template <typename F>
void parallel_for(int64_t n, F f) {
  int nt = num_threads();
  if (n < 100000) nt = 1;
  std::vector<std::thread> th;
  th.reserve((size_t)nt);  // may throw, before any thread exists
  int64_t per = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    int64_t b = t * per, e = std::min<int64_t>(n, b + per);
    if (b >= e) break;
    bool started = false;
    if (t > 0) {  // chunk 0 runs here, after the others have started
      try {
        th.emplace_back([=] { f(b, e, t); });
        started = true;
      } catch (...) {
      }
    }
    if (!started && t > 0) f(b, e, t);
  }
  if (n > 0) f(0, std::min<int64_t>(n, per), 0);
  for (auto &x : th) x.join();
}

// Runs a host builder, turning an allocation failure (or another C++
// exception of the standard library) into a status: none crosses the C ABI.
template <typename F>
int host_guard(F f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    return APSPIE_ERR_OOM;
  } catch (const std::exception &) {
    return APSPIE_ERR_INVALID;
  }
}

// LSD radix sort of 64-bit keys on the low `bits` bits, 11-bit digits.
void radix_sort_u64(std::vector<uint64_t> &a, int bits) {
  const int64_t n = (int64_t)a.size();
  if (n < 2) return;
  std::vector<uint64_t> tmp(n);
  const int D = 11, R = 1 << D;
  int nt = num_threads();  // as parallel_for: one histogram per chunk
  if (n < 100000) nt = 1;
  std::vector<int64_t> hist((size_t)nt * R);
  uint64_t *src = a.data(), *dst = tmp.data();
  int passes = 0;
  for (int shift = 0; shift < bits; shift += D, ++passes) {
    std::fill(hist.begin(), hist.end(), 0);
    // parallel_for's chunks are the ones `per` describes: chunk t counts
    // into and scatters from histogram t
    parallel_for(n, [&](int64_t b, int64_t e, int t) {
      int64_t *h = &hist[(size_t)t * R];
      for (int64_t i = b; i < e; ++i) h[(src[i] >> shift) & (R - 1)]++;
    });
    int64_t run = 0;
    for (int d = 0; d < R; ++d)
      for (int t = 0; t < nt; ++t) {
        int64_t c = hist[(size_t)t * R + d];
        hist[(size_t)t * R + d] = run;
        run += c;
      }
    parallel_for(n, [&](int64_t b, int64_t e, int t) {
      int64_t *h = &hist[(size_t)t * R];
      for (int64_t i = b; i < e; ++i) dst[h[(src[i] >> shift) & (R - 1)]++] = src[i];
    });
    std::swap(src, dst);
  }
  if (passes & 1) a.swap(tmp);
}

// Sorted, deduplicated (row<<32|col) keys -> CSR.  Keys equal to ~0 are
// padding and are dropped (they sort last).
int keys_to_csr(std::vector<uint64_t> &keys, int m, int64_t *nnz_out, int **h_ptr,
                int **h_ind) {
  int64_t n = (int64_t)keys.size();
  while (n > 0 && keys[n - 1] == ~0ull) --n;
  int64_t w = 0;
  for (int64_t i = 0; i < n; ++i)
    if (i == 0 || keys[i] != keys[i - 1]) keys[w++] = keys[i];
  if (w >= (int64_t)INT32_MAX) return APSPIE_ERR_OVERFLOW;
  int *ptr = (int *)malloc(sizeof(int) * ((size_t)m + 1));
  int *ind = (int *)malloc(sizeof(int) * (size_t)(w > 0 ? w : 1));
  if (!ptr || !ind) {
    free(ptr);
    free(ind);
    return APSPIE_ERR_OOM;
  }
  std::memset(ptr, 0, sizeof(int) * ((size_t)m + 1));
  for (int64_t i = 0; i < w; ++i) ptr[(keys[i] >> 32) + 1]++;
  for (int i = 0; i < m; ++i) ptr[i + 1] += ptr[i];
  parallel_for(w, [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; ++i) ind[i] = (int)(keys[i] & 0xffffffffu);
  });
  *nnz_out = w;
  *h_ptr = ptr;
  *h_ind = ind;
  return APSPIE_OK;
}

int bits_for(int m) {
  int b = 0;
  while ((1ll << b) < (long long)m) ++b;
  return b;
}

}  // namespace

using namespace apspie_gen;

extern "C" {

int apspie_gen_rmat_host(int scale, int edge_factor, uint64_t seed, int symmetric,
                         int scramble, int *m_out, int64_t *nnz_out, int **h_ptr,
                         int **h_ind) {
  return host_guard([&]() -> int {
    if (scale < 1 || scale > 30 || edge_factor < 1 || !m_out || !nnz_out || !h_ptr || !h_ind)
      return APSPIE_ERR_INVALID;
    const int m = 1 << scale;
    const int64_t samples = (int64_t)edge_factor << scale;
    const int per = symmetric ? 2 : 1;
    std::vector<uint64_t> keys((size_t)(samples * per));
    const RmatParams P = rmat_params(scale, seed, scramble != 0);
    parallel_for(samples, [&](int64_t b, int64_t e, int) {
      for (int64_t s = b; s < e; ++s) {
        uint32_t u, v;
        rmat_sample(P, (uint64_t)s, &u, &v);
        if (u == v) {
          keys[(size_t)(s * per)] = ~0ull;
          if (symmetric) keys[(size_t)(s * per + 1)] = ~0ull;
        } else {
          keys[(size_t)(s * per)] = ((uint64_t)u << 32) | v;
          if (symmetric) keys[(size_t)(s * per + 1)] = ((uint64_t)v << 32) | u;
        }
      }
    });
    // pad keys (~0) must sort last: sort on all 64 bits only when needed
    radix_sort_u64(keys, 32 + scale + (1));
    *m_out = m;
    return keys_to_csr(keys, m, nnz_out, h_ptr, h_ind);
  });
}

int apspie_gen_er_host(int n, int mean_degree, uint64_t seed, int64_t *nnz_out, int **h_ptr,
                       int **h_ind) {
  return host_guard([&]() -> int {
    if (n < 2 || mean_degree < 1 || !nnz_out || !h_ptr || !h_ind) return APSPIE_ERR_INVALID;
    const int64_t samples = (int64_t)n * mean_degree / 2;
    std::vector<uint64_t> keys((size_t)(2 * samples));
    const uint64_t sm = mix64(seed ^ 0x45524552ull);
    parallel_for(samples, [&](int64_t b, int64_t e, int) {
      for (int64_t s = b; s < e; ++s) {
        uint32_t u, v;
        er_sample(sm, (uint64_t)s, (uint32_t)n, &u, &v);
        if (u == v) {
          keys[(size_t)(2 * s)] = keys[(size_t)(2 * s + 1)] = ~0ull;
        } else {
          keys[(size_t)(2 * s)] = ((uint64_t)u << 32) | v;
          keys[(size_t)(2 * s + 1)] = ((uint64_t)v << 32) | u;
        }
      }
    });
    radix_sort_u64(keys, 32 + bits_for(n) + 1);
    return keys_to_csr(keys, n, nnz_out, h_ptr, h_ind);
  });
}

int apspie_gen_grid_host(int rows, int cols, int64_t *nnz_out, int **h_ptr, int **h_ind) {
  if (rows < 1 || cols < 1 || (int64_t)rows * cols >= INT32_MAX || !nnz_out || !h_ptr || !h_ind)
    return APSPIE_ERR_INVALID;
  const int m = rows * cols;
  int *ptr = (int *)malloc(sizeof(int) * ((size_t)m + 1));
  int64_t nnz = 4ll * rows * cols - 2ll * rows - 2ll * cols;
  int *ind = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
  if (!ptr || !ind) {
    free(ptr);
    free(ind);
    return APSPIE_ERR_OOM;
  }
  int64_t k = 0;
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) {
      ptr[r * cols + c] = (int)k;
      // neighbours in ascending id order: up, left, right, down
      if (r > 0) ind[k++] = (r - 1) * cols + c;
      if (c > 0) ind[k++] = r * cols + c - 1;
      if (c + 1 < cols) ind[k++] = r * cols + c + 1;
      if (r + 1 < rows) ind[k++] = (r + 1) * cols + c;
    }
  ptr[m] = (int)k;
  *nnz_out = k;
  *h_ptr = ptr;
  *h_ind = ind;
  return APSPIE_OK;
}

int apspie_gen_weights_u32_host(int m, const int *h_ptr, const int *h_ind, uint64_t seed,
                                uint32_t lo, uint32_t hi, uint32_t *h_w) {
  return host_guard([&]() -> int {
    if (m < 0 || !h_ptr || !h_w || hi < lo) return APSPIE_ERR_INVALID;
    parallel_for(m, [&](int64_t b, int64_t e, int) {
      for (int64_t u = b; u < e; ++u)
        for (int k = h_ptr[u]; k < h_ptr[u + 1]; ++k)
          h_w[k] = weight_u32(seed, (uint32_t)u, (uint32_t)h_ind[k], lo, hi);
    });
    return APSPIE_OK;
  });
}

int apspie_gen_weights_f32_host(int m, const int *h_ptr, const int *h_ind, uint64_t seed,
                                float *h_w) {
  return host_guard([&]() -> int {
    if (m < 0 || !h_ptr || !h_w) return APSPIE_ERR_INVALID;
    parallel_for(m, [&](int64_t b, int64_t e, int) {
      for (int64_t u = b; u < e; ++u)
        for (int k = h_ptr[u]; k < h_ptr[u + 1]; ++k)
          h_w[k] = weight_f32(seed, (uint32_t)u, (uint32_t)h_ind[k]);
    });
    return APSPIE_OK;
  });
}

int apspie_mt19937_fill_host(uint32_t seed, int64_t n, uint32_t *h_out) {
  if (n < 0 || (n > 0 && !h_out)) return APSPIE_ERR_INVALID;
  uint32_t mt[624];
  int mti;
  mt[0] = seed;
  for (mti = 1; mti < 624; ++mti)
    mt[mti] = 1812433253u * (mt[mti - 1] ^ (mt[mti - 1] >> 30)) + (uint32_t)mti;
  for (int64_t t = 0; t < n; ++t) {
    if (mti >= 624) {
      // twist: the first 227 words read words not yet updated in this pass,
      // the rest read already-updated ones
      for (int k = 0; k < 624; ++k) {
        uint32_t y = (mt[k] & 0x80000000u) | (mt[k + 1 < 624 ? k + 1 : 0] & 0x7fffffffu);
        uint32_t src = mt[k + 397 < 624 ? k + 397 : k + 397 - 624];
        mt[k] = src ^ (y >> 1) ^ ((y & 1u) * 0x9908b0dfu);
      }
      mti = 0;
    }
    uint32_t y = mt[mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    h_out[t] = y;
  }
  return APSPIE_OK;
}

// Mean of floor(X) for X ~ Pareto(alpha, xmin) truncated at T (continuous).
static double powerlaw_floor_mean(double alpha, double xmin, double T, int max_deg) {
  double tail = std::pow(xmin / T, alpha - 1.0);
  double mean = 0.0;
  for (int k = 1; k <= max_deg; ++k) {
    double p = (double)k <= xmin ? 1.0 : (std::pow(xmin / k, alpha - 1.0) - tail) / (1.0 - tail);
    if (p <= 0) break;
    mean += p;
  }
  return mean;
}

int apspie_gen_powerlaw_host(int m, int n, double alpha, double mean, int max_deg, uint64_t seed,
                             double *xmin_out, int64_t *nnz_out, int **h_ptr, int **h_ind,
                             float **h_val) {
  return host_guard([&]() -> int {
    if (m < 1 || n < 1 || alpha <= 1.0 || mean < 1.0 || max_deg < 1 || !nnz_out || !h_ptr ||
        !h_ind || !h_val)
      return APSPIE_ERR_INVALID;
    const double T = (double)max_deg + 1.0;
    // x_min such that E[floor(X)] = mean, by bisection
    double lo = 1.0, hi = (double)max_deg;
    for (int it = 0; it < 200; ++it) {
      double mid = 0.5 * (lo + hi);
      if (powerlaw_floor_mean(alpha, mid, T, max_deg) < mean) lo = mid; else hi = mid;
    }
    const double xmin = 0.5 * (lo + hi);
    if (xmin_out) *xmin_out = xmin;
    const double tail = std::pow(xmin / T, alpha - 1.0);
    const uint64_t sd = mix64(seed ^ 0x504c4157ull);
    std::vector<int> k((size_t)m);
    parallel_for(m, [&](int64_t b, int64_t e, int) {
      for (int64_t i = b; i < e; ++i) {
        // u uniform in (0, 1]; inverse CDF of the truncated Pareto
        double u = ((double)(mix64(sd ^ (uint64_t)i) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
        double x = xmin * std::pow(1.0 - u * (1.0 - tail), -1.0 / (alpha - 1.0));
        int d = (int)std::floor(x);
        k[(size_t)i] = std::max(1, std::min(d, std::min(max_deg, n)));
      }
    });
    std::vector<int64_t> off((size_t)m + 1, 0);
    for (int i = 0; i < m; ++i) off[(size_t)i + 1] = off[(size_t)i] + k[(size_t)i];
    std::vector<int> cols((size_t)off[(size_t)m]);
    std::vector<int> cnt((size_t)m);
    parallel_for(m, [&](int64_t b, int64_t e, int) {
      for (int64_t i = b; i < e; ++i) {
        int *c = cols.data() + off[(size_t)i];
        int ki = k[(size_t)i];
        for (int t = 0; t < ki; ++t) {
          uint64_t h = mix64(mix64(sd ^ 0xC01ull ^ ((uint64_t)i << 20)) ^ (uint64_t)t);
          c[t] = (int)(((h & 0xffffffffull) * (uint64_t)n) >> 32);
        }
        std::sort(c, c + ki);
        cnt[(size_t)i] = (int)(std::unique(c, c + ki) - c);
      }
    });
    int64_t nnz = 0;
    for (int i = 0; i < m; ++i) nnz += cnt[(size_t)i];
    if (nnz >= (int64_t)INT32_MAX) return APSPIE_ERR_OVERFLOW;
    int *ptr = (int *)malloc(sizeof(int) * ((size_t)m + 1));
    int *ind = (int *)malloc(sizeof(int) * (size_t)std::max<int64_t>(1, nnz));
    float *val = (float *)malloc(sizeof(float) * (size_t)std::max<int64_t>(1, nnz));
    if (!ptr || !ind || !val) {
      free(ptr);
      free(ind);
      free(val);
      return APSPIE_ERR_OOM;
    }
    ptr[0] = 0;
    for (int i = 0; i < m; ++i) ptr[i + 1] = ptr[i] + cnt[(size_t)i];
    parallel_for(m, [&](int64_t b, int64_t e, int) {
      for (int64_t i = b; i < e; ++i) {
        const int *c = cols.data() + off[(size_t)i];
        for (int t = 0; t < cnt[(size_t)i]; ++t) {
          int p = ptr[i] + t;
          ind[p] = c[t];
          uint64_t h = mix64(mix64(sd ^ 0x7A1ull) ^ (((uint64_t)i << 32) | (uint32_t)c[t]));
          val[p] = (float)((double)(h >> 40) * (1.0 / 8388608.0) - 1.0);  // k*2^-23 - 1 in [-1, 1)
        }
      }
    });
    *nnz_out = nnz;
    *h_ptr = ptr;
    *h_ind = ind;
    *h_val = val;
    return APSPIE_OK;
  });
}

void apspie_host_free(void *p) { free(p); }

}  // extern "C"
