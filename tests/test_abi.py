"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(apspie_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from apspie_b200 import _native
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    # the Python binding declares a prototype for each of them too
    assert not (names - set(_native.PROTOS)), sorted(names - set(_native.PROTOS))


def test_status_strings_and_null_context():
    from apspie_b200._native import lib
    assert lib.apspie_status_string(0) == b"ok"
    assert lib.apspie_status_string(4) == b"device-side wait timed out"
    # calls on a null context return an error instead of crashing
    assert lib.apspie_ctx_sync(None) == 1
    assert lib.apspie_bfs(None, 0, 0, 1, None, None, None, None, None, 0) == 1


def test_library_is_built_for_sm_100a():
    """The build recipe targets sm_100a only (no PTX for other targets)."""
    from apspie_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-lineinfo" in build.COMMON

def test_ctypes_structs_match_the_header_layout(tmp_path):
    """The Python binding's struct mirrors have the C header's sizes and
    field offsets (compiled here with gcc against include/apspie.h)."""
    import shutil
    import subprocess
    import pytest
    from apspie_b200 import _native as N
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = {"apspie_tuning": N.Tuning, "apspie_job": N.Job, "apspie_bfs_stats": N.BfsStats,
             "apspie_sssp_stats": N.SsspStats, "apspie_csr": N.Csr,
             "apspie_batch_stats": N.BatchStats, "apspie_server_stats": N.ServerStats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "apspie.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in pairs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_python_constants_match_the_header_enums(tmp_path):
    """The enum values the Python binding and the tests use (semirings, job
    types, statuses, test-hook codes) are the header's (compiled with gcc)."""
    import shutil
    import subprocess
    import pytest
    from apspie_b200 import ops
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    names = ["APSPIE_PLUS_TIMES", "APSPIE_MIN_PLUS", "APSPIE_MAX_TIMES", "APSPIE_OR_AND",
             "APSPIE_JOB_BFS", "APSPIE_JOB_SSSP_U32", "APSPIE_ERR_OOM", "APSPIE_ERR_CUDA",
             "APSPIE_ERR_TIMEOUT", "APSPIE_ERR_TOO_LARGE", "APSPIE_INJECT_BFS_BARRIER",
             "APSPIE_INJECT_SORT_LOOKBACK", "APSPIE_INJECT_ALLOC_FAIL"]
    src = tmp_path / "enums.c"
    src.write_text('#include <stdio.h>\n#include "apspie.h"\nint main(void) {\n' +
                   "".join(f'  printf("{n} %d\\n", (int){n});\n' for n in names) +
                   "  return 0;\n}\n")
    exe = tmp_path / "enums"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {l.split()[0]: int(l.split()[1]) for l in out.splitlines() if l.strip()}
    assert (got["APSPIE_PLUS_TIMES"], got["APSPIE_MIN_PLUS"], got["APSPIE_MAX_TIMES"],
            got["APSPIE_OR_AND"]) == (ops.PLUS_TIMES, ops.MIN_PLUS, ops.MAX_TIMES, ops.OR_AND)
    assert (got["APSPIE_JOB_BFS"], got["APSPIE_JOB_SSSP_U32"]) == (ops.JOB_BFS, ops.JOB_SSSP_U32)
    # the values tests/test_failures.py and tests/test_zz_no_alloc.py spell out
    assert (got["APSPIE_ERR_OOM"], got["APSPIE_ERR_CUDA"], got["APSPIE_ERR_TIMEOUT"],
            got["APSPIE_ERR_TOO_LARGE"]) == (2, 3, 4, 8)
    assert (got["APSPIE_INJECT_BFS_BARRIER"], got["APSPIE_INJECT_SORT_LOOKBACK"],
            got["APSPIE_INJECT_ALLOC_FAIL"]) == (1, 2, 3)
