"""Python binding of the oracle (the CPU checker) and of the reference's own
CPU routines compiled into oracle/_ref/.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, never by the apspie_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libapspie_ref.so"


def build() -> None:
    """make -C oracle (compiles the reference routines too when the reference
    tree is present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


if not ORACLE_SO.exists():
    build()

_o = C.CDLL(str(ORACLE_SO))
_r = C.CDLL(str(REF_SO)) if REF_SO.exists() else None

vp, ci, i64 = C.c_void_p, C.c_int, C.c_int64
_o.orc_bfs.argtypes = [ci, vp, vp, ci, ci, vp]
_o.orc_bfs.restype = ci
for _n in ("orc_sssp_f32", "orc_sssp_f64", "orc_sssp_u32"):
    getattr(_o, _n).argtypes = [ci, vp, vp, vp, ci, vp]
    getattr(_o, _n).restype = None
_o.orc_mis.argtypes = [ci, vp, vp, vp, vp]
_o.orc_neighbor_flags.argtypes = [ci, vp, vp, vp, vp]
_o.orc_mis_check.argtypes = [ci, vp, vp, vp]
_o.orc_mis_check.restype = ci
_o.orc_tc_build_lower.argtypes = [ci, vp, vp, vp, vp, vp]
_o.orc_tc_build_lower.restype = ci
_o.orc_tc_lower.argtypes = [ci, vp, vp]
_o.orc_tc_lower.restype = i64
_o.orc_spgemm_symbolic.argtypes = [ci, ci, vp, vp, vp, vp, vp]
_o.orc_spgemm_symbolic.restype = i64
_o.orc_spgemm_numeric.argtypes = [ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, vp]
_o.orc_spmspv.argtypes = [ci, ci, vp, vp, vp, ci, vp, vp, vp, vp]
_o.orc_spmspv.restype = ci
_o.orc_mt_fill.argtypes = [C.c_uint32, i64, vp]
if _r is not None:
    _r.ref_bfs_cpu.argtypes = [ci, ci, vp, vp, vp, ci]
    _r.ref_bfs_cpu.restype = ci
    _r.ref_sssp_cpu.argtypes = [ci, ci, vp, vp, vp, vp, ci]
    _r.ref_sssp_cpu.restype = ci
    _r.ref_mt_fill.argtypes = [C.c_ulong, C.c_longlong, vp]
    _r.ref_tc_ewise.argtypes = [ci, i64, vp, vp, vp, vp, vp, vp, vp]
    _r.ref_tc_ewise.restype = None
    _r.ref_mis.argtypes = [ci, vp, vp, vp, C.c_float, vp]
    _r.ref_mis.restype = ci

PLUS_TIMES, MIN_PLUS, MAX_TIMES, OR_AND = 0, 1, 2, 3


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


def _d(x):
    return x.ctypes.data if x is not None and x.size else None


def have_reference() -> bool:
    return _r is not None


# ------------------------------------------------------------- oracle ---
def bfs(m, ptr, ind, src, stop=1 << 30):
    ptr, ind = _a(ptr, np.int32), _a(ind, np.int32)
    d = np.empty(m, dtype=np.int32)
    depth = _o.orc_bfs(m, _d(ptr), _d(ind), src, stop, _d(d))
    return d, depth


def sssp_f32(m, ptr, ind, w, src):
    d = np.empty(m, dtype=np.float32)
    _o.orc_sssp_f32(m, _d(_a(ptr, np.int32)), _d(_a(ind, np.int32)), _d(_a(w, np.float32)), src,
                    _d(d))
    return d


def sssp_f64(m, ptr, ind, w, src):
    d = np.empty(m, dtype=np.float64)
    _o.orc_sssp_f64(m, _d(_a(ptr, np.int32)), _d(_a(ind, np.int32)), _d(_a(w, np.float32)), src,
                    _d(d))
    return d


def sssp_u32(m, ptr, ind, w, src):
    d = np.empty(m, dtype=np.uint32)
    _o.orc_sssp_u32(m, _d(_a(ptr, np.int32)), _d(_a(ind, np.int32)), _d(_a(w, np.uint32)), src,
                    _d(d))
    return d


def mis(m, ptr, ind, prio):
    out = np.empty(m, dtype=np.int32)
    _o.orc_mis(m, _d(_a(ptr, np.int32)), _d(_a(ind, np.int32)), _d(_a(prio, np.uint32)), _d(out))
    return out


def neighbor_flags(m, ptr, ind, flags):
    out = np.empty(m, dtype=np.int32)
    _o.orc_neighbor_flags(m, _d(_a(ptr, np.int32)), _d(_a(ind, np.int32)),
                          _d(_a(flags, np.int32)), _d(out))
    return out


def mis_check(m, ptr, ind, mis_vec) -> int:
    return int(_o.orc_mis_check(m, _d(_a(ptr, np.int32)), _d(_a(ind, np.int32)),
                                _d(_a(mis_vec, np.int32))))


def tc_build_lower(m, ptr, ind):
    ptr, ind = _a(ptr, np.int32), _a(ind, np.int32)
    perm = np.empty(m, dtype=np.int32)
    lp = np.empty(m + 1, dtype=np.int32)
    li = np.empty(max(1, ind.size // 2 + 1), dtype=np.int32)
    n = _o.orc_tc_build_lower(m, _d(ptr), _d(ind), _d(perm), _d(lp), _d(li))
    return perm, lp, li[:n].copy()


def tc_lower(m, lp, li) -> int:
    return int(_o.orc_tc_lower(m, _d(_a(lp, np.int32)), _d(_a(li, np.int32))))


def spgemm(m, n, ap, ai, av, bp, bi, bv):
    ap, ai, bp, bi = (_a(x, np.int32) for x in (ap, ai, bp, bi))
    av = None if av is None else _a(av, np.float32)
    bv = None if bv is None else _a(bv, np.float32)
    cp = np.empty(m + 1, dtype=np.int64)
    nnz = _o.orc_spgemm_symbolic(m, n, _d(ap), _d(ai), _d(bp), _d(bi), _d(cp))
    cind = np.empty(max(1, nnz), dtype=np.int32)
    cval = np.empty(max(1, nnz), dtype=np.float64)
    _o.orc_spgemm_numeric(m, n, _d(ap), _d(ai), _d(av), _d(bp), _d(bi), _d(bv), _d(cp),
                          _d(cind), _d(cval))
    return cp, cind[:nnz].copy(), cval[:nnz].copy()


def spmspv(semiring, m, ptr, ind, val, xind, xval):
    ptr, ind = _a(ptr, np.int32), _a(ind, np.int32)
    val = None if val is None else _a(val, np.float32)
    xind = _a(xind, np.int32)
    xval = None if xval is None else _a(xval, np.float32)
    yi = np.empty(max(1, m), dtype=np.int32)
    yv = np.empty(max(1, m), dtype=np.float64)
    n = _o.orc_spmspv(semiring, m, _d(ptr), _d(ind), _d(val), xind.size, _d(xind), _d(xval),
                      _d(yi), _d(yv))
    return yi[:n].copy(), yv[:n].copy()


def mt_fill(seed, n):
    out = np.empty(n, dtype=np.uint32)
    _o.orc_mt_fill(seed, n, _d(out))
    return out


# ---------------------------------------------- the reference's own code ---
def _quiet(fn, *args):
    """The reference routines print timings to stdout; keep them out of the
    caller's stdout (bench.py prints exactly one JSON line)."""
    import sys
    sys.stdout.flush()
    C.CDLL(None).fflush(None)
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(devnull, 1)
        return fn(*args)
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def ref_bfs(m, ptr, ind, src, stop=1 << 30):
    ptr, ind = _a(ptr, np.int32), _a(ind, np.int32)
    d = np.empty(m, dtype=np.int32)
    depth = _quiet(_r.ref_bfs_cpu, src, m, _d(ptr), _d(ind), _d(d), stop)
    return d, depth


def ref_sssp(m, ptr, ind, w, src):
    ptr, ind = _a(ptr, np.int32), _a(ind, np.int32)
    d = np.empty(m, dtype=np.float32)
    _quiet(_r.ref_sssp_cpu, src, m, _d(ptr), _d(ind), _d(_a(w, np.float32)), _d(d), 1 << 30)
    return d


def ref_mt_fill(seed, n):
    out = np.empty(n, dtype=np.uint32)
    _r.ref_mt_fill(seed, n, _d(out))
    return out


def ref_tc(m, ptr, ind) -> int:
    """Triangles of a symmetric graph by the reference's own
    intersection kernel ewiseMultTc (src/tc.cuh:168-199, built host-side in
    oracle/_ref), fed as test/tc/main.cu:172-175,241-244 feed it: C = the
    strictly upper part and B = the strictly lower part in CSC (self-loops
    fall in neither, as in buildLower, test/tc/main.cu:40-55), D = the
    product that cuSPARSE csrgemm forms from C's and B's arrays (computed
    here by the oracle's Gustavson SpGEMM), then the per-thread counts summed
    (mgpu::Reduce, test/tc/main.cu:247) in int64."""
    ptr, ind = _a(ptr, np.int64), _a(ind, np.int64)
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(ptr))

    def part(keep):
        r, c = rows[keep], ind[keep]
        order = np.lexsort((c, r))
        p = np.zeros(m + 1, np.int64)
        np.add.at(p, r + 1, 1)
        return np.cumsum(p).astype(np.int32), c[order].astype(np.int32)

    cp, ci_ = part(ind < rows)   # column i of C (CSC): rows j < i
    bp, bi = part(ind > rows)    # column i of B (CSC): rows j > i
    dp, di, dv = spgemm(m, m, cp, ci_, None, bp, bi, None)
    dp32 = dp.astype(np.int32)
    # one readable entry past the end of each row index array (the kernel
    # reads it when a column is exhausted, src/tc.cuh:190,194)
    di_pad = np.append(di.astype(np.int32), np.int32(0))
    ci_pad = np.append(ci_, np.int32(0))
    dv = _a(dv, np.float64)
    cv = np.ones(max(1, ci_.size), np.float64)
    nthreads = ((m + 511) // 512) * 512
    out = np.zeros(max(1, nthreads), np.float64)
    _r.ref_tc_ewise(m, int(di.size), _d(dv), _d(dp32), _d(di_pad), _d(cv), _d(cp), _d(ci_pad),
                    _d(out))
    return int(np.sum(out[:m].astype(np.int64)))


def ref_mis(m, ptr, ind, prio_u32, delta: float):
    """MIS by the reference's own round kernels (src/spmspvMis.cuh:10-78,
    built host-side in oracle/_ref) driven by its round loop
    (src/spmspvMis.cuh:232-318), with the uint32 priorities mapped to
    prio / 2^32 in double (same order, every value below 1 as the
    reference's fillUniform draws are).  Returns (membership 1 / 0 / -1,
    rounds)."""
    ptr, ind = _a(ptr, np.int32), _a(ind, np.int32)
    pr = _a(prio_u32, np.uint32).astype(np.float64) / 4294967296.0
    out = np.empty(m, dtype=np.int32)
    rounds = _r.ref_mis(m, _d(ptr), _d(ind), _d(pr), float(delta), _d(out))
    return out, int(rounds)
