// gen_common.h -- counter-based random draws shared by the host and device
// graph builders, so both produce the same edge multiset bit for bit.
//
// mix64 is the splitmix64 finaliser (Steele, Lea & Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014).  All thresholds are
// integers, so no floating point enters the edge choice.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define APSPIE_HD __host__ __device__ __forceinline__
#else
#define APSPIE_HD inline
#endif

namespace apspie_gen {

APSPIE_HD uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// R-MAT quadrant thresholds: floor(p * 2^32) for the cumulative
// probabilities 0.57, 0.76, 0.95 of (a, a+b, a+b+c).
constexpr uint32_t kRmatA = 2448131358u;
constexpr uint32_t kRmatAB = 3264175144u;
constexpr uint32_t kRmatABC = 4080218931u;

struct RmatParams {
  int scale;
  uint64_t seed;  // mixed seed
  uint64_t mask;
  uint64_t k1, k2, k3;  // scramble constants (k1, k3 odd)
  int scramble;
};

APSPIE_HD RmatParams rmat_params(int scale, uint64_t seed, bool scramble) {
  RmatParams p;
  p.scale = scale;
  p.seed = mix64(seed ^ 0x524d4154ull);
  p.mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
  p.k1 = (mix64(p.seed ^ 1) | 1ull) & p.mask;
  p.k2 = mix64(p.seed ^ 2) & p.mask;
  p.k3 = (mix64(p.seed ^ 3) | 1ull) & p.mask;
  p.scramble = scramble ? 1 : 0;
  return p;
}

// Bijection on [0, 2^scale): odd multiply + add, xorshift, odd multiply,
// xorshift -- each step is invertible modulo 2^scale.
APSPIE_HD uint32_t rmat_scramble(const RmatParams &p, uint64_t x) {
  x = (x * p.k1 + p.k2) & p.mask;
  x ^= x >> (p.scale / 2 + 1);
  x = (x * p.k3) & p.mask;
  x ^= x >> (p.scale / 3 + 1);
  return (uint32_t)x;
}

// Sample s of the R-MAT edge stream: one 32-bit draw per recursion level,
// two levels per splitmix64 output, most significant bit first.
APSPIE_HD void rmat_sample(const RmatParams &p, uint64_t s, uint32_t *u, uint32_t *v) {
  uint64_t r = 0, c = 0;
  uint64_t draw = 0;
  for (int l = 0; l < p.scale; ++l) {
    if ((l & 1) == 0) draw = mix64(p.seed ^ ((s << 5) | (uint64_t)(l >> 1)));
    uint32_t x = (l & 1) ? (uint32_t)(draw >> 32) : (uint32_t)draw;
    uint64_t rb = x >= kRmatAB;                       // quadrants c, d
    uint64_t cb = (x >= kRmatA && x < kRmatAB) || x >= kRmatABC;  // b, d
    r = (r << 1) | rb;
    c = (c << 1) | cb;
  }
  if (p.scramble) {
    r = rmat_scramble(p, r);
    c = rmat_scramble(p, c);
  }
  *u = (uint32_t)r;
  *v = (uint32_t)c;
}

// Erdos-Renyi pair: two 32-bit draws mapped to [0, n) by multiply-shift.
APSPIE_HD void er_sample(uint64_t mixed_seed, uint64_t s, uint32_t n, uint32_t *u, uint32_t *v) {
  uint64_t d = mix64(mixed_seed ^ s);
  *u = (uint32_t)(((d & 0xffffffffull) * n) >> 32);
  *v = (uint32_t)(((d >> 32) * n) >> 32);
}

APSPIE_HD uint32_t weight_u32(uint64_t seed, uint32_t u, uint32_t v, uint32_t lo, uint32_t hi) {
  uint64_t h = mix64(mix64(seed ^ 0x57454947ull) ^ (((uint64_t)u << 32) | v));
  uint64_t span = (uint64_t)hi - lo + 1;
  return lo + (uint32_t)(h % span);
}

// (k + 1) * 2^-24 for k in [0, 2^24): uniform on (0, 1], exact in float.
APSPIE_HD float weight_f32(uint64_t seed, uint32_t u, uint32_t v) {
  uint64_t h = mix64(mix64(seed ^ 0x46333257ull) ^ (((uint64_t)u << 32) | v));
  return (float)((h >> 40) + 1) * (1.0f / 16777216.0f);
}

}  // namespace apspie_gen
