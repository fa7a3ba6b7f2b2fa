"""Generate tests/golden/golden.npz from the reference's own CPU code.

Runs in a checkout that has the reference tree (the environment variable
REF_ROOT, required, names its root) and the compiled reference routines
(oracle/_ref, built by `make -C oracle REF_SRC=$REF_ROOT/src`).  The output is committed; tests read only the .npz.

Contents
  mtx/<name>/{dir,und}_{ptr,ind}   CSR of each dataset/small/*.mtx file, parsed
                                   here with the reference's orientation (row =
                                   2nd index, col = 1st, src/util.cuh:382-386),
                                   undirected = makeSymmetric (util.cuh:573-643)
  mtx/<name>/{dir,und}_bfs         bfsCPU depth from every source, shape (m, m)
  mtx/<name>/und_w, und_sssp       per-edge float weights and ssspCPU distances
                                   from every source (reference output, -1 =
                                   unreached)
  mt/5489, mt/42                   first 2000 genrand_int32 outputs
  rmat10/*                         BFS / SSSP of the reference on R-MAT scale 10
                                   graphs from the package's generator, plus a
                                   SHA-256 of each CSR (pins the generator)
  tc/<name>                        triangle count of each undirected fixture and
                                   of R-MAT 10 / 12 (symmetrised, seed 3) by the
                                   reference's ewiseMultTc built host-side
                                   (oracle.ref_tc)
  mis/<name>/ptr, ind              self-loop-free symmetric graphs (the
                                   undirected fixtures, R-MAT 10, ER 2^10 mean
                                   degree 8, a 24x24 grid)
  mis/<name>/d<delta>, rounds_*    MIS membership (1 / 0) and rounds from the
                                   reference's round kernels and loop
                                   (oracle.ref_mis) with mt19937(5489)
                                   priorities, delta 0.1 and 1
"""
from __future__ import annotations

import hashlib
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import oracle  # noqa: E402

if "REF_ROOT" not in os.environ:
    raise SystemExit("make_golden.py: set REF_ROOT to the root of the apspie source tree")
REF_ROOT = Path(os.environ["REF_ROOT"])
FIXTURES = ["test_cc", "test_bc", "test_pr", "test_spgemm", "test_mis", "test_mesh", "chesapeake"]


def parse_mtx(path: Path):
    """Return (m, rows, cols) with row = second index, col = first index."""
    rows, cols = [], []
    m = None
    with open(path) as f:
        for line in f:
            if line.startswith("%"):
                continue
            parts = line.split()
            if not parts:
                continue
            if m is None:
                m = int(parts[0])
                continue
            cols.append(int(parts[0]) - 1)
            rows.append(int(parts[1]) - 1)
    return m, np.array(rows, np.int64), np.array(cols, np.int64)


def csr(m, rows, cols):
    order = np.argsort(rows, kind="stable")
    ptr = np.zeros(m + 1, np.int64)
    np.add.at(ptr, rows + 1, 1)
    return np.cumsum(ptr).astype(np.int32), cols[order].astype(np.int32)


def symmetrise(rows, cols):
    keep = rows != cols
    r = np.concatenate([rows, cols[keep]])
    c = np.concatenate([cols, rows[keep]])
    key = np.unique(r * (1 << 32) + c)
    return key >> 32, key & 0xffffffff


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def weights(ptr, ind):
    # deterministic per-edge float weights in (0, 1] on the 2^-8 grid
    src = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    return (((src * 131 + ind * 71) % 256) + 1).astype(np.float32) / 256.0


def main() -> None:
    assert oracle.have_reference(), "build oracle/_ref first (make -C oracle)"
    out: dict[str, np.ndarray] = {}
    for name in FIXTURES:
        m, rows, cols = parse_mtx(REF_ROOT / "dataset" / "small" / f"{name}.mtx")
        for kind, (r, c) in (("dir", (rows, cols)), ("und", symmetrise(rows, cols))):
            ptr, ind = csr(m, r, c)
            out[f"mtx/{name}/{kind}_ptr"] = ptr
            out[f"mtx/{name}/{kind}_ind"] = ind
            out[f"mtx/{name}/{kind}_bfs"] = np.stack(
                [oracle.ref_bfs(m, ptr, ind, s)[0] for s in range(m)])
            if kind == "und":
                w = weights(ptr, ind)
                out[f"mtx/{name}/und_w"] = w
                out[f"mtx/{name}/und_sssp"] = np.stack(
                    [oracle.ref_sssp(m, ptr, ind, w, s) for s in range(m)])
    out["mt/5489"] = oracle.ref_mt_fill(5489, 2000)
    out["mt/42"] = oracle.ref_mt_fill(42, 2000)

    import apspie_b200 as ap
    g = ap.gen_rmat(10, 16, seed=3, symmetric=True)
    out["rmat10/sym_sha"] = np.frombuffer(sha(g.ptr, g.ind).encode(), np.uint8)
    srcs = np.array(ap.seeded_sources(g, 3, seed=1), np.int32)
    out["rmat10/sym_src"] = srcs
    out["rmat10/sym_bfs"] = np.stack([oracle.ref_bfs(g.m, g.ptr, g.ind, int(s))[0] for s in srcs])
    gd = ap.gen_rmat(10, 16, seed=3, symmetric=False)
    wu = ap.weights_u32(gd, seed=11)
    wf = ap.weights_f32(gd, seed=11)
    out["rmat10/dir_sha"] = np.frombuffer(sha(gd.ptr, gd.ind, wu, wf).encode(), np.uint8)
    out["rmat10/dir_sssp_u32"] = np.stack(
        [oracle.ref_sssp(gd.m, gd.ptr, gd.ind, wu.astype(np.float32), int(s)) for s in srcs])
    out["rmat10/dir_sssp_f32"] = np.stack(
        [oracle.ref_sssp(gd.m, gd.ptr, gd.ind, wf, int(s)) for s in srcs])
    # triangle counts by the reference's intersection kernel
    for name in FIXTURES:
        ptr, ind = out[f"mtx/{name}/und_ptr"], out[f"mtx/{name}/und_ind"]
        out[f"tc/{name}"] = np.array([oracle.ref_tc(len(ptr) - 1, ptr, ind)], np.int64)
    for sc in (10, 12):
        gt = ap.gen_rmat(sc, 16, seed=3, symmetric=True)
        out[f"tc/rmat{sc}"] = np.array([oracle.ref_tc(gt.m, gt.ptr, gt.ind)], np.int64)
    # MIS by the reference's round kernels, on graphs without self-loops
    # (a self-looped vertex never joins the reference's set)
    mis_graphs = {}
    for name in FIXTURES:
        ptr, ind = out[f"mtx/{name}/und_ptr"], out[f"mtx/{name}/und_ind"]
        m = len(ptr) - 1
        rows = np.repeat(np.arange(m), np.diff(ptr))
        mis_graphs[name] = csr(m, rows[rows != ind], ind[rows != ind].astype(np.int64))
    gm = ap.gen_rmat(10, 16, seed=3, symmetric=True)
    mis_graphs["rmat10"] = (gm.ptr, gm.ind)
    ge = ap.gen_er(1 << 10, 8, seed=3)
    mis_graphs["er10"] = (ge.ptr, ge.ind)
    gg = ap.gen_grid(24, 24)
    mis_graphs["grid24"] = (gg.ptr, gg.ind)
    for name, (ptr, ind) in mis_graphs.items():
        m = len(ptr) - 1
        prio = oracle.ref_mt_fill(5489, m)
        out[f"mis/{name}/ptr"] = np.asarray(ptr, np.int32)
        out[f"mis/{name}/ind"] = np.asarray(ind, np.int32)
        for delta in (0.1, 1.0):
            mis, rounds = oracle.ref_mis(m, ptr, ind, prio, delta)
            assert np.all(mis >= 0), f"{name}: undecided vertices"
            out[f"mis/{name}/d{delta}"] = mis.astype(np.int8)
            out[f"mis/{name}/rounds_d{delta}"] = np.array([rounds], np.int32)
    np.savez_compressed(Path(__file__).with_name("golden.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
