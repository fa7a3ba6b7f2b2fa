"""The reference-facing C++ API (include/apspie_ref.hpp): a driver written
against the reference's signatures compiles against the library (CPU) and
reports CORRECT on every fixture and algorithm (GPU)."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "ref_api_main.cpp"
CUDA = Path("/usr/local/cuda")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    import oracle  # noqa: F401  (builds oracle/liboracle.so if needed)
    out = tmp_path_factory.mktemp("cpp") / "ref_api_main"
    lib = ROOT / "apspie_b200" / "_lib"
    cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{ROOT / 'oracle'}",
           f"-I{CUDA / 'include'}", str(SRC), "-o", str(out),
           f"-L{lib}", "-lapspie_b200", f"-L{ROOT / 'oracle'}", "-l:liboracle.so",
           f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{lib}", f"-Wl,-rpath,{ROOT / 'oracle'}", f"-Wl,-rpath,{CUDA / 'lib64'}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return out


def test_driver_compiles_against_the_reference_api(driver):
    assert driver.exists()


def _write_mtx(path, ptr, ind):
    m = len(ptr) - 1
    rows = np.repeat(np.arange(m), np.diff(ptr))
    with open(path, "w") as f:
        f.write(f"{m} {m} {len(ind)}\n")
        for r, c in zip(rows, ind):
            f.write(f"{c + 1} {r + 1}\n")


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["bfs", "spmspvbfs", "sssp", "mis", "mxv", "spmv", "csr2csc",
                                  "spgemm", "spgemm_csc", "mxm", "tc"])
def test_driver_correct_on_fixtures(driver, golden, fixture_names, tmp_path, algo):
    for name in fixture_names:
        path = tmp_path / f"{name}.mtx"
        _write_mtx(path, golden[f"mtx/{name}/dir_ptr"], golden[f"mtx/{name}/dir_ind"])
        args = [str(driver), algo, str(path), "-source", "1"]
        if algo in ("mis", "tc", "bfs"):
            args.append("-undirected")
        if algo in ("mis", "tc") and name == "test_spgemm":
            continue  # self-loops: a looped vertex is its own neighbour in the flag check
        res = subprocess.run(args, capture_output=True, text=True, timeout=120)
        assert res.returncode == 0, f"{name}: {res.stdout}\n{res.stderr}"
        assert "CORRECT" in res.stdout and "INCORRECT" not in res.stdout


CHECKS_SRC = r"""
#include <cstdio>
#include <cstdlib>
#include "apspie_ref.hpp"
// buildMatrix refuses COO entries outside the matrix before it writes a host
// array or touches the device (so this runs without a GPU).
static int expect_invalid(d_matrix *A, int n, int *r, int *c, float *v) {
  try {
    buildMatrix<float>(A, n, r, c, v);
  } catch (const apspie::Error &e) {
    return e.status == APSPIE_ERR_INVALID ? 0 : 1;
  }
  return 1;
}
int main() {
  d_matrix A;
  A.m = 3;
  A.n = 3;
  A.h_cscColPtr = (int *)calloc(4, sizeof(int));
  int r0[2] = {0, 3}, c0[2] = {1, 1};     // row 3 of 3
  int r1[1] = {0}, c1[1] = {-1};          // column -1
  int r2[1] = {-2}, c2[1] = {0};          // row -2
  int r3[1] = {2}, c3[1] = {3};           // column 3 of 3
  float v[2] = {1.0f, 1.0f};
  int bad = expect_invalid(&A, 2, r0, c0, v) + expect_invalid(&A, 1, r1, c1, v) +
            expect_invalid(&A, 1, r2, c2, v) + expect_invalid(&A, 1, r3, c3, v);
  free(A.h_cscColPtr);
  printf(bad ? "FAILED\n" : "ok\n");
  return bad;
}
"""


def test_build_matrix_refuses_entries_outside_the_matrix(tmp_path):
    """The shim's buildMatrix indexes host arrays by the caller's COO rows;
    entries outside [0, m) x [0, n) raise apspie::Error(APSPIE_ERR_INVALID)
    instead of writing past them."""
    src = tmp_path / "checks.cpp"
    src.write_text(CHECKS_SRC)
    out = tmp_path / "checks"
    cmd = ["g++", "-O1", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}",
           str(src), "-o", str(out), f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{CUDA / 'lib64'}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    run = subprocess.run([str(out)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
