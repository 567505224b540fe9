"""ctypes binding of the C ABI in ``include/sj/sj_join.h`` (``sirius_b200/libsj.so``).

There is no fallback: if the library is missing or does not load, importing the join API
raises, so a GPU run can never silently take a CPU or library path.
"""
from __future__ import annotations

import ctypes
from ctypes import (POINTER, Structure, c_double, c_float, c_int32, c_int64, c_size_t, c_uint32, c_uint64, c_void_p,
                    c_char_p, CFUNCTYPE)
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsj.so"

# sj_status
SJ_OK, SJ_ERR_OOM, SJ_ERR_TABLE_FULL, SJ_ERR_INVALID, SJ_ERR_DEVICE, SJ_ERR_TIMEOUT, SJ_ERR_CAPACITY, \
    SJ_ERR_BUSY = range(8)
# sj_type
SJ_INT8, SJ_INT16, SJ_INT32, SJ_INT64, SJ_FLOAT32, SJ_FLOAT64, SJ_BOOL8, SJ_UINT32, SJ_UINT64 = range(1, 10)
# layouts / null equality / slot kinds
SJ_LAYOUT_AUTO, SJ_LAYOUT_DISTINCT, SJ_LAYOUT_GROUPED = 0, 1, 2
SJ_NULLS_UNEQUAL, SJ_NULLS_EQUAL = 0, 1
SJ_SLOT_PACKED64, SJ_SLOT_WIDE128 = 0, 1
SJ_AGG_AUTO, SJ_AGG_WARP, SJ_AGG_CTA, SJ_AGG_WARP_DYNAMIC = 0, 1, 2, 3
SJ_JOIN_INNER, SJ_JOIN_LEFT, SJ_JOIN_SEMI, SJ_JOIN_ANTI, SJ_JOIN_MARK, SJ_JOIN_FULL = range(6)
SJ_NO_ROW = -(1 << 31)
SJ_PROBE_KERNEL_AUTO, SJ_PROBE_KERNEL_STAGED, SJ_PROBE_KERNEL_DIRECT, SJ_PROBE_KERNEL_DIRECT_TMA = 0, 1, 2, 3
SJ_L2_AUTO, SJ_L2_NORMAL, SJ_L2_EVICT_LAST = 0, 1, 2


class SjColumn(Structure):
    _fields_ = [("data", c_void_p), ("validity", c_void_p), ("validity_offset", c_int64),
                ("num_rows", c_int64), ("type", c_int32), ("reserved", c_int32)]


class SjMutColumn(Structure):
    _fields_ = [("data", c_void_p), ("validity", c_void_p), ("type", c_int32), ("reserved", c_int32)]


ALLOC_FN = CFUNCTYPE(c_void_p, c_void_p, c_size_t, c_void_p)
FREE_FN = CFUNCTYPE(None, c_void_p, c_void_p, c_size_t, c_void_p)


class SjAlloc(Structure):
    _fields_ = [("ctx", c_void_p), ("alloc", ALLOC_FN), ("free", FREE_FN)]


class SjJoinParams(Structure):
    _fields_ = [("layout", c_int32), ("null_equality", c_int32), ("load_factor", c_float),
                ("block_size", c_int32), ("group_width", c_int32), ("partition_bits", c_int32),
                ("force_wide", c_int32), ("ctas_per_sm", c_int32), ("aggregation", c_int32),
                ("probe_kernel", c_int32), ("rows_per_lane", c_int32), ("probe_partition_mb", c_int32),
                ("table_l2_priority", c_int32), ("bloom_bits_per_key", c_int32), ("reserved", c_int32 * 2)]


class SjTableInfo(Structure):
    _fields_ = [("build_rows", c_int64), ("valid_rows", c_int64), ("null_rows", c_int64),
                ("distinct_keys", c_int64), ("num_slots", c_int64), ("device_bytes", c_int64),
                ("key_min", c_int64), ("key_max", c_int64), ("layout", c_int32), ("slot_kind", c_int32),
                ("rid_bits", c_int32), ("key_type", c_int32), ("partition_bits", c_int32),
                ("max_group", c_int32)]


class SjBatchJoin(Structure):
    _fields_ = [("build_key", SjColumn), ("build_payload", SjColumn), ("probe_key", SjColumn),
                ("probe_payload", SjColumn), ("out_probe_rid", c_void_p), ("out_build_rid", c_void_p),
                ("out_probe_payload", SjMutColumn), ("out_build_payload", SjMutColumn), ("capacity", c_int64)]


class SjBatchParams(Structure):
    _fields_ = [("block_size", c_int32), ("group_width", c_int32), ("load_factor", c_float),
                ("tile_rows", c_int32), ("ctas_per_sm", c_int32), ("reserved", c_int32 * 7)]


class SjKernelTime(Structure):
    _fields_ = [("name", c_char_p), ("ms", c_float), ("reserved", c_int32)]


class SjServerConfig(Structure):
    _fields_ = [("slots", c_int32), ("max_skip", c_int32), ("memory_budget_bytes", c_int64),
                ("reserve_bytes", c_int64), ("batch_small", c_int32), ("reserved", c_int32 * 5)]


class SjRequestResult(Structure):
    _fields_ = [("request_id", c_uint64), ("status", c_int32), ("table_id", c_int32), ("count", c_int64),
                ("probe_rows", c_int64), ("probe_rid", c_void_p), ("build_rid", c_void_p),
                ("build_payload", c_void_p * 8), ("build_validity", c_void_p * 8), ("t_submit", c_double),
                ("t_admit", c_double), ("t_done", c_double)]


# (name, restype, argtypes) of every function the header declares.
_P = POINTER
SIGNATURES = {
    "sj_default_params": (None, [_P(SjJoinParams)]),
    "sj_build": (c_int32, [_P(SjColumn), c_int32, _P(SjJoinParams), _P(SjAlloc), c_void_p, _P(c_void_p)]),
    "sj_build_ex": (c_int32, [_P(SjColumn), c_int32, _P(SjColumn), c_int32, _P(SjJoinParams), _P(SjAlloc), c_void_p,
                              _P(c_void_p)]),
    "sj_table_destroy": (c_int32, [c_void_p, c_void_p]),
    "sj_table_get_info": (c_int32, [c_void_p, _P(SjTableInfo)]),
    "sj_probe_count": (c_int32, [c_void_p, _P(SjColumn), c_int32, _P(SjAlloc), c_void_p, c_void_p]),
    "sj_probe_gather": (c_int32, [c_void_p, _P(SjColumn), c_int32, _P(SjColumn), c_int32, _P(SjColumn), c_int32,
                                  c_void_p, c_void_p, _P(SjMutColumn), _P(SjMutColumn), c_int64, _P(SjAlloc),
                                  c_void_p, c_void_p]),
    "sj_inner_join": (c_int32, [_P(SjColumn), _P(SjColumn), c_int32, _P(SjColumn), c_int32, _P(SjColumn), c_int32,
                                c_void_p, c_void_p, _P(SjMutColumn), _P(SjMutColumn), c_int64, _P(SjJoinParams),
                                _P(SjAlloc), c_void_p, c_void_p]),
    "sj_inner_join_host": (c_int32, [_P(SjColumn), _P(SjColumn), c_int32, _P(SjColumn), c_int32, _P(SjColumn),
                                     c_int32, c_void_p, c_void_p, _P(SjMutColumn), _P(SjMutColumn), c_int64, c_int64,
                                     _P(SjJoinParams), _P(SjAlloc), c_void_p, _P(c_int64)]),
    "sj_inner_join_noalloc": (c_int32, [_P(SjColumn), _P(SjColumn), c_int32, _P(SjColumn), c_int32, _P(SjColumn),
                                        c_int32, c_void_p, c_void_p, _P(SjMutColumn), _P(SjMutColumn), c_int64,
                                        _P(SjJoinParams), c_void_p, c_void_p]),
    "sj_probe_join": (c_int32, [c_void_p, c_int32, _P(SjColumn), c_int32, _P(SjColumn), c_int32, _P(SjColumn),
                                c_int32, c_void_p, c_void_p, _P(SjMutColumn), _P(SjMutColumn), c_int64, c_void_p,
                                c_void_p, _P(SjAlloc), c_void_p, c_void_p]),
    "sj_hash_partition": (c_int32, [_P(SjColumn), c_int32, _P(SjColumn), c_int32, c_int32, _P(SjMutColumn),
                                    c_void_p, _P(SjAlloc), c_void_p]),
    "sj_bloom_build": (c_int32, [_P(SjColumn), c_int32, _P(SjAlloc), c_void_p, _P(c_void_p)]),
    "sj_bloom_contains": (c_int32, [c_void_p, _P(SjColumn), c_void_p, c_void_p, c_void_p]),
    "sj_bloom_bytes": (c_int64, [c_void_p]),
    "sj_table_bloom": (c_void_p, [c_void_p]),
    "sj_bloom_destroy": (c_int32, [c_void_p, c_void_p]),
    "sj_status_string": (c_char_p, [c_int32]),
    "sj_last_error": (c_char_p, []),
    "sj_version": (c_int32, []),
    "sj_debug_wait_timeout": (c_int32, [c_int32, c_void_p, c_void_p]),
    "sj_timing_enable": (None, [c_int32]),
    "sj_batch_plan_create": (c_int32, [_P(SjBatchJoin), c_int32, _P(SjBatchParams), _P(SjAlloc), c_void_p,
                                       _P(c_void_p)]),
    "sj_batch_plan_launch": (c_int32, [c_void_p, c_void_p]),
    "sj_batch_plan_replay": (c_int32, [c_void_p, c_void_p]),
    "sj_batch_plan_launch_per_join": (c_int32, [c_void_p, c_void_p]),
    "sj_batch_plan_counts": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "sj_batch_plan_destroy": (c_int32, [c_void_p, c_void_p]),
    "sj_timing_collect": (c_int32, [_P(SjKernelTime), c_int32]),
    "sj_server_create": (c_int32, [_P(SjServerConfig), _P(c_void_p)]),
    "sj_server_add_table": (c_int32, [c_void_p, _P(SjColumn), _P(SjColumn), c_int32, _P(SjJoinParams), _P(c_int32)]),
    "sj_server_submit": (c_int32, [c_void_p, c_int32, _P(SjColumn), c_uint64]),
    "sj_server_poll": (c_int32, [c_void_p, _P(SjRequestResult), c_int32, c_int32]),
    "sj_server_release": (c_int32, [c_void_p, c_uint64]),
    "sj_server_destroy": (c_int32, [c_void_p]),
}

_lib = None


class SjError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: {status_name(status)}: {message}")


def load(path: Path | str | None = None):
    """Load libsj.so (raises OSError / FileNotFoundError if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run __graft_entry__.build() (no CPU fallback exists)")
    L = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = L
    return L


def status_name(s: int) -> str:
    try:
        return load().sj_status_string(s).decode()
    except Exception:  # pragma: no cover
        return str(s)


def check(status: int, where: str):
    if status != SJ_OK:
        L = load()
        raise SjError(status, where, L.sj_last_error().decode())


def default_params(**overrides) -> SjJoinParams:
    p = SjJoinParams()
    load().sj_default_params(ctypes.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def timing_enable(on: bool = True):
    load().sj_timing_enable(int(on))


def timing_collect(capacity: int = 4096):
    """[(kernel name, ms)] recorded on this thread since the last collect (waits for the events)."""
    buf = (SjKernelTime * capacity)()
    n = load().sj_timing_collect(buf, capacity)
    return [(buf[i].name.decode(), float(buf[i].ms)) for i in range(min(n, capacity))]
