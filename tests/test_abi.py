"""The C ABI library loads on a CPU-only machine, exports every function the headers declare,
and its struct layouts match both the C compiler's and the ctypes binding's. No GPU calls."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include" / "sj").glob("*.h"))
DECL = re.compile(r"SJ_EXPORT\s+[\w\s\*]+?\b(sj_\w+)\s*\(", re.S)


def declared():
    names = []
    for h in HEADERS:
        names += DECL.findall(h.read_text())
    return sorted(set(names))


def test_headers_declare_functions():
    names = declared()
    assert "sj_build" in names and "sj_probe_gather" in names
    assert len(names) >= 10


def test_every_declared_symbol_is_exported(built):
    from sirius_b200 import _lib
    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_every_declared_symbol(built):
    from sirius_b200 import _lib
    assert set(declared()) <= set(_lib.SIGNATURES) | set(getattr(_lib, "EXTRA_SIGNATURES", {}))


def test_exports_are_only_the_abi(built):
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "sirius_b200" / "libsj.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = sorted({l.split()[-1] for l in out.splitlines() if " T " in l})
    assert all(s.startswith("sj_") for s in exported), exported


def test_struct_layout_matches_c(built, tmp_path):
    from sirius_b200 import _lib
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "sj/sj_join.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(sj_column), sizeof(sj_mut_column), sizeof(sj_alloc),
         sizeof(sj_join_params), sizeof(sj_table_info));
  printf("%zu %zu %zu\n", offsetof(sj_column, num_rows), offsetof(sj_join_params, ctas_per_sm),
         offsetof(sj_table_info, max_group));
  printf("%zu %zu %zu %zu %zu\n", sizeof(sj_batch_join), sizeof(sj_batch_params), sizeof(sj_kernel_time),
         sizeof(sj_server_config), sizeof(sj_request_result));
  printf("%zu %zu %zu\n", offsetof(sj_batch_join, capacity), offsetof(sj_request_result, build_validity),
         offsetof(sj_request_result, t_done));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    exp = [ctypes.sizeof(_lib.SjColumn), ctypes.sizeof(_lib.SjMutColumn), ctypes.sizeof(_lib.SjAlloc),
           ctypes.sizeof(_lib.SjJoinParams), ctypes.sizeof(_lib.SjTableInfo),
           _lib.SjColumn.num_rows.offset, _lib.SjJoinParams.ctas_per_sm.offset, _lib.SjTableInfo.max_group.offset,
           ctypes.sizeof(_lib.SjBatchJoin), ctypes.sizeof(_lib.SjBatchParams), ctypes.sizeof(_lib.SjKernelTime),
           ctypes.sizeof(_lib.SjServerConfig), ctypes.sizeof(_lib.SjRequestResult),
           _lib.SjBatchJoin.capacity.offset, _lib.SjRequestResult.build_validity.offset,
           _lib.SjRequestResult.t_done.offset]
    assert [int(x) for x in got] == exp


def test_host_only_calls(built):
    from sirius_b200 import _lib
    lib = _lib.load()
    p = _lib.default_params()
    assert abs(p.load_factor - 0.5) < 1e-6 and p.layout == _lib.SJ_LAYOUT_AUTO
    assert lib.sj_status_string(_lib.SJ_ERR_OOM) == b"SJ_ERR_OOM"
    assert lib.sj_version() >= 100


def test_argument_validation_needs_no_gpu(built):
    """Bad arguments are rejected before any CUDA call."""
    from sirius_b200 import _lib
    lib = _lib.load()
    col = _lib.SjColumn()
    col.type = _lib.SJ_INT32
    out = ctypes.c_void_p()
    st = lib.sj_build(ctypes.byref(col), 5, None, None, None, ctypes.byref(out))
    assert st == _lib.SJ_ERR_INVALID
    assert b"1 to 4 key columns" in lib.sj_last_error()
    col.type = _lib.SJ_FLOAT32
    st = lib.sj_build(ctypes.byref(col), 1, None, None, None, ctypes.byref(out))
    assert st == _lib.SJ_ERR_INVALID
    assert b"INT32 or INT64" in lib.sj_last_error()
    st = lib.sj_build(ctypes.byref(col), 1, None, None, None, None)
    assert st == _lib.SJ_ERR_INVALID
    with pytest.raises(_lib.SjError):
        _lib.check(_lib.SJ_ERR_INVALID, "x")


def test_host_join_argument_validation_needs_no_gpu(built):
    """sj_inner_join_host refuses payloads with NULLs, key-type mismatches and missing outputs before
    any CUDA call."""
    import numpy as np
    from sirius_b200 import _lib
    lib = _lib.load()
    keys = np.arange(64, dtype=np.int64)
    words = np.full(2, -1, dtype=np.int32)

    def col(a, valid=None):
        c = _lib.SjColumn()
        c.data = a.ctypes.data
        c.validity = valid.ctypes.data if valid is not None else None
        c.num_rows = len(a)
        c.type = _lib.SJ_INT64 if a.dtype == np.int64 else _lib.SJ_INT32
        return c
    cnt = ctypes.c_int64(-1)
    pay = (_lib.SjColumn * 1)(col(keys, words))
    out = (_lib.SjMutColumn * 1)()
    st = lib.sj_inner_join_host(ctypes.byref(col(keys)), ctypes.byref(col(keys)), 1, pay, 1, None, 0, None, None,
                                out, None, 0, 0, None, None, None, ctypes.byref(cnt))
    assert st == _lib.SJ_ERR_INVALID and b"payload columns with NULLs" in lib.sj_last_error()
    k32 = np.arange(64, dtype=np.int32)
    st = lib.sj_inner_join_host(ctypes.byref(col(keys)), ctypes.byref(col(k32)), 1, None, 0, None, 0, None, None,
                                None, None, 0, 0, None, None, None, ctypes.byref(cnt))
    assert st == _lib.SJ_ERR_INVALID and b"key types differ" in lib.sj_last_error()
    pay = (_lib.SjColumn * 1)(col(keys))
    st = lib.sj_inner_join_host(ctypes.byref(col(keys)), ctypes.byref(col(keys)), 1, pay, 1, None, 0, None, None,
                                None, None, 64, 0, None, None, None, ctypes.byref(cnt))
    assert st == _lib.SJ_ERR_INVALID and b"output missing" in lib.sj_last_error()


def test_library_missing_fails_loudly(tmp_path):
    from sirius_b200 import _lib
    with pytest.raises(FileNotFoundError):
        _lib.load(tmp_path / "nope.so")
