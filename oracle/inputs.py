"""Benchmark inputs built without the apspie_b200 library: a NumPy
restatement of its host R-MAT builder and of its source choice, so the
reference arm of bench.py times the reference's CPU BFS on the same graph and
sources while loading none of the product's code.

TEST INFRASTRUCTURE ONLY (bench.py's reference arm and the tests that pin
this restatement to the library's builder bit for bit).

The builder: sample s of the R-MAT edge stream draws one 32-bit value per
recursion level, two levels per splitmix64 output (Steele, Lea & Flood,
OOPSLA 2014) of seed' ^ (s << 5 | level / 2), most significant level first;
the quadrant thresholds are floor(p * 2^32) of the cumulative probabilities
0.57, 0.76, 0.95; vertex ids go through a seeded bijection (odd multiply and
add, xorshift, odd multiply, xorshift modulo 2^scale); self-loops are
dropped, the graph is optionally symmetrised, (row, col) pairs are sorted
and deduplicated into CSR.
"""
from __future__ import annotations

import numpy as np

_A, _AB, _ABC = np.uint64(2448131358), np.uint64(3264175144), np.uint64(4080218931)


def _mix64(z):
    """splitmix64 finaliser on a uint64 array (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _mix1(x: int) -> int:
    return int(_mix64(np.array([x], dtype=np.uint64))[0])


def _scramble(x, scale, k1, k2, k3, mask):
    with np.errstate(over="ignore"):
        x = (x * k1 + k2) & mask
        x ^= x >> np.uint64(scale // 2 + 1)
        x = (x * k3) & mask
        x ^= x >> np.uint64(scale // 3 + 1)
    return x


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 1, symmetric: bool = True,
             scramble: bool = True, chunk: int = 1 << 23):
    """(m, ptr int32[m+1], ind int32[nnz]) equal to apspie_gen_rmat_host."""
    m = 1 << scale
    samples = edge_factor << scale
    pseed = _mix1(seed ^ 0x524D4154)
    mask = (1 << scale) - 1
    k1 = np.uint64((_mix1(pseed ^ 1) | 1) & mask)
    k2 = np.uint64(_mix1(pseed ^ 2) & mask)
    k3 = np.uint64((_mix1(pseed ^ 3) | 1) & mask)
    mk, ps = np.uint64(mask), np.uint64(pseed)
    parts = []
    for b in range(0, samples, chunk):
        s = np.arange(b, min(samples, b + chunk), dtype=np.uint64)
        r = np.zeros_like(s)
        c = np.zeros_like(s)
        for lv in range(scale):
            if lv % 2 == 0:
                draw = _mix64(ps ^ ((s << np.uint64(5)) | np.uint64(lv >> 1)))
            x = (draw >> np.uint64(32)) if lv % 2 else (draw & np.uint64(0xFFFFFFFF))
            rb = (x >= _AB).astype(np.uint64)
            cb = (((x >= _A) & (x < _AB)) | (x >= _ABC)).astype(np.uint64)
            r = (r << np.uint64(1)) | rb
            c = (c << np.uint64(1)) | cb
        if scramble:
            r = _scramble(r, scale, k1, k2, k3, mk)
            c = _scramble(c, scale, k1, k2, k3, mk)
        keep = r != c
        r, c = r[keep], c[keep]
        parts.append((r << np.uint64(32)) | c)
        if symmetric:
            parts.append((c << np.uint64(32)) | r)
    key = np.concatenate(parts)
    del parts
    key.sort()
    first = np.empty(len(key), dtype=bool)
    first[:1] = True
    np.not_equal(key[1:], key[:-1], out=first[1:])
    key = key[first]
    rows = (key >> np.uint64(32)).astype(np.int64)
    ind = (key & np.uint64(0xFFFFFFFF)).astype(np.int32)
    ptr = np.zeros(m + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.bincount(rows, minlength=m))
    return m, ptr.astype(np.int32), ind


def seeded_sources(m: int, ptr, ind, k: int, seed: int = 0) -> list[int]:
    """k seed-chosen vertices of the largest (weakly) connected component,
    drawn as apspie_b200.seeded_sources draws them."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    a = sp.csr_matrix((np.ones(len(ind), dtype=np.int8), ind, ptr), shape=(m, m))
    _, label = connected_components(a, directed=True, connection="weak")
    members = np.flatnonzero(label == int(np.argmax(np.bincount(label))))
    rng = np.random.default_rng(seed)
    return [int(x) for x in members[rng.integers(len(members), size=k)]]
