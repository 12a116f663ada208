"""ctypes binding of the C ABI in ``include/mordred_b200.h``.

The library is the in-tree ``libmordred_b200.so`` built by :mod:`mordred_b200.build`.
Loading never falls back to anything else: if the library is missing or does not
load, :func:`lib` raises, so no query can silently run off the GPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

# ---- constants (mirror include/mordred_b200.h) -------------------------------------
MB_OK = 0
MB_ERR_ARG, MB_ERR_ALIGN, MB_ERR_LAUNCH, MB_ERR_CUDA, MB_ERR_NODEV, MB_ERR_SIZE = 1, 2, 3, 4, 5, 6
MB_STATUS_PROBE_RANGE = 0x1
MB_STATUS_GROUP_RANGE = 0x2
MB_STATUS_TIMEOUT = 0x4
MB_STATUS_OVERFLOW = 0x8

MB_FILTER_EQ, MB_FILTER_BETWEEN, MB_FILTER_EQ_OR_EQ = 0, 1, 2
MB_HT_KEY, MB_HT_KEY_VAL, MB_HT_VAL_OFF, MB_HT_PASS = 0, 1, 2, 3
MB_AGG_SUM, MB_AGG_SUB, MB_AGG_MUL, MB_AGG_MUL_PAYLOAD = 0, 1, 2, 3
MB_RES_SCALAR, MB_RES_ENGINE6, MB_RES_CRYSTAL4, MB_RES_DENSE = 0, 1, 2, 3
MB_MAX_FILTERS, MB_MAX_PROBES = 3, 4

# generator column ids (mordred_b200/csrc/ssbgen.h)
MB_LO_ORDERDATE, MB_LO_QUANTITY, MB_LO_DISCOUNT, MB_LO_EXTENDEDPRICE = 0, 1, 2, 3
MB_LO_SUPPKEY, MB_LO_CUSTKEY, MB_LO_PARTKEY, MB_LO_REVENUE, MB_LO_SUPPLYCOST = 4, 5, 6, 7, 8
MB_D_DATEKEY, MB_D_YEAR, MB_D_YEARMONTHNUM = 16, 17, 18
MB_S_SUPPKEY, MB_S_CITY, MB_S_NATION, MB_S_REGION = 32, 33, 34, 35
MB_C_CUSTKEY, MB_C_CITY, MB_C_NATION, MB_C_REGION = 48, 49, 50, 51
MB_P_PARTKEY, MB_P_BRAND1, MB_P_CATEGORY, MB_P_MFGR = 64, 65, 66, 67


class MbFilter(C.Structure):
    _fields_ = [("col", C.c_void_p), ("mode", C.c_int), ("c1", C.c_int), ("c2", C.c_int)]


class MbProbe(C.Structure):
    _fields_ = [("fkey", C.c_void_p), ("ht", C.c_void_p), ("num_slots", C.c_int),
                ("key_min", C.c_int), ("layout", C.c_int), ("min_val", C.c_int),
                ("unique_val", C.c_int), ("res_slot", C.c_int), ("presence", C.c_void_p)]


class MbStarArgs(C.Structure):
    _fields_ = [("num_rows", C.c_int64), ("num_filters", C.c_int),
                ("filter", MbFilter * MB_MAX_FILTERS), ("num_probes", C.c_int),
                ("probe", MbProbe * MB_MAX_PROBES), ("aggr", C.c_void_p * 2),
                ("agg_op", C.c_int), ("total_val", C.c_int), ("group_bias", C.c_int),
                ("res_layout", C.c_int), ("res", C.c_void_p), ("count", C.c_void_p),
                ("count_after", C.c_int), ("gpu_cache", C.c_void_p),
                ("segment_group", C.c_void_p), ("start_offset", C.c_int64),
                ("segment_size", C.c_int), ("threads", C.c_int),
                ("items_per_thread", C.c_int), ("stages", C.c_int), ("grid", C.c_int),
                ("group_mode", C.c_int), ("rows", C.c_void_p), ("mirrors", C.c_int),
                ("pack", C.c_int)]


class MbFilterArgsGPU(C.Structure):
    _fields_ = [("filter_idx1", C.c_void_p), ("filter_idx2", C.c_void_p),
                ("compare1", C.c_int), ("compare2", C.c_int), ("compare3", C.c_int),
                ("compare4", C.c_int), ("mode1", C.c_int), ("mode2", C.c_int)]


class MbProbeArgsGPU(C.Structure):
    _fields_ = ([(f"key_idx{i}", C.c_void_p) for i in range(1, 5)]
                + [(f"ht{i}", C.c_void_p) for i in range(1, 5)]
                + [(f"dim_len{i}", C.c_int) for i in range(1, 5)]
                + [(f"min_key{i}", C.c_int) for i in range(1, 5)])


class MbGroupbyArgsGPU(C.Structure):
    _fields_ = ([("aggr_idx1", C.c_void_p), ("aggr_idx2", C.c_void_p)]
                + [(f"group_idx{i}", C.c_void_p) for i in range(1, 5)]
                + [(f"min_val{i}", C.c_int) for i in range(1, 5)]
                + [(f"unique_val{i}", C.c_int) for i in range(1, 5)]
                + [("total_val", C.c_int), ("mode", C.c_int)])


class MbBuildArgsGPU(C.Structure):
    _fields_ = [("key_idx", C.c_void_p), ("val_idx", C.c_void_p), ("num_slots", C.c_int),
                ("val_min", C.c_int), ("val_max", C.c_int)]


P = C.c_void_p
I = C.c_int
I64 = C.c_int64
U64 = C.c_uint64
PS = C.POINTER

# name -> (restype, argtypes); every symbol declared in include/mordred_b200.h
SIGNATURES = {
    "mb_star_query": (I, [PS(MbStarArgs), P]),
    "mb_build_pht": (I, [P, I, I, I, P, P, I, P, I, I, P, P]),
    "mb_join_build": (I, [P, P, I, P, I, P]),
    "mb_join_probe": (I, [P, P, I, P, I, P, P]),
    "mb_q11_query": (I, [P, P, P, P, I, P, P, P]),
    "mb_q21_probe": (I, [P, P, P, P, I, P, I, P, I, P, I, P, P]),
    "mb_q41_probe": (I, [P, P, P, P, P, P, I, P, I, P, I, P, I, P, I, P, P]),
    "mb_q41_probe_noalloc": (I, [P, P, P, P, P, P, I, P, I, P, I, P, I, P, I, P, P, P]),
    "mb_filter_probe_group_by_GPU2": (I, [P, PS(MbFilterArgsGPU), PS(MbProbeArgsGPU),
                                          PS(MbGroupbyArgsGPU), I, P, I, P, P]),
    "mb_probe_group_by_GPU2": (I, [P, PS(MbProbeArgsGPU), PS(MbGroupbyArgsGPU), I, P, I, P, P]),
    "mb_filter_probe_aggr_GPU2": (I, [P, PS(MbFilterArgsGPU), PS(MbProbeArgsGPU),
                                      PS(MbGroupbyArgsGPU), I, P, I, P, P]),
    "mb_build_GPU2": (I, [P, PS(MbFilterArgsGPU), PS(MbBuildArgsGPU), I, P, I, P, P]),
    "mb_gen_fact_column": (I, [I, U64, I64, I64, I, I, I, P, P]),
    "mb_gen_dim_column": (I, [I, U64, I64, P, P]),
    "mb_gen_fact_column_host": (I, [I, U64, I64, I64, I, I, I, P, I]),
    "mb_gen_dim_column_host": (I, [I, U64, I64, P, I]),
    "mb_version": (I, []),
    "mb_init": (I, [I]),
    "mb_device_status": (I, [I, PS(C.c_uint), I]),
    "mb_error_string": (C.c_char_p, [I]),
    "mb_launch_count": (C.c_ulonglong, []),
    "mb_device_state_ready": (I, [I]),
}


class MbError(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed: {msg} (code {code})")
        self.code = code


_lock = threading.Lock()
_lib: C.CDLL | None = None


def lib_path() -> str:
    return _build.LIB


def lib() -> C.CDLL:
    """Load (building first if the sources are newer) and return the library."""
    global _lib
    with _lock:
        if _lib is None:
            path = lib_path()
            if not os.path.exists(path) or not _build.up_to_date():
                # a library older than its sources is never used: rebuild or fail
                try:
                    _build.build()
                except Exception as e:
                    raise ImportError(f"libmordred_b200.so is missing or stale and the build failed: {e}")
            l = C.CDLL(path)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(l, name)
                fn.restype = res
                fn.argtypes = args
            _lib = l
        return _lib


def check(name: str, code: int) -> None:
    if code != MB_OK:
        msg = lib().mb_error_string(code).decode()
        raise MbError(name, code, msg)


def call(name: str, *args) -> None:
    check(name, getattr(lib(), name)(*args))


def device_status(device: int = -1, clear: bool = True) -> int:
    st = C.c_uint(0)
    call("mb_device_status", device, C.byref(st), 1 if clear else 0)
    return st.value


def launch_count() -> int:
    return int(lib().mb_launch_count())


# ---- batched multi-query (include/mordred_b200.h) ------------------------------------
MB_BATCH_MAX_QUERIES, MB_BATCH_MAX_PREDS = 256, 4
(MB_COL_ORDERDATE, MB_COL_QUANTITY, MB_COL_DISCOUNT, MB_COL_EXTENDEDPRICE, MB_COL_SUPPKEY, MB_COL_CUSTKEY,
 MB_COL_PARTKEY, MB_COL_REVENUE, MB_COL_SUPPLYCOST, MB_COL_DIM_S, MB_COL_DIM_C, MB_COL_DIM_P,
 MB_COL_DIM_D) = range(13)
MB_NUM_FACT_COLS = 9


def MB_FIELD(col: int, shift: int, width: int) -> int:
    return (col << 11) | (shift << 6) | width


class MbPat(C.Structure):
    _fields_ = [("words", C.c_void_p), ("slots", C.c_int), ("key_min", C.c_int)]


class MbBatchQuery(C.Structure):
    _fields_ = [("num_preds", C.c_int), ("pred_field", C.c_int * MB_BATCH_MAX_PREDS),
                ("pred_lo", C.c_int * MB_BATCH_MAX_PREDS), ("pred_hi", C.c_int * MB_BATCH_MAX_PREDS),
                ("dims_required", C.c_int), ("agg_op", C.c_int), ("agg_field", C.c_int * 2),
                ("num_keys", C.c_int), ("key_field", C.c_int * 2), ("key_min", C.c_int * 2),
                ("key_mul", C.c_int * 2), ("total_val", C.c_int), ("res_layout", C.c_int), ("res", C.c_void_p)]


class MbBatchArgs(C.Structure):
    _fields_ = [("num_rows", C.c_int64), ("fact", C.c_void_p * MB_NUM_FACT_COLS), ("dim", MbPat * 4),
                ("num_queries", C.c_int), ("queries", C.POINTER(MbBatchQuery)), ("workspace", C.c_void_p),
                ("workspace_bytes", C.c_size_t), ("threads", C.c_int), ("items_per_thread", C.c_int),
                ("stages", C.c_int), ("grid", C.c_int), ("smem_group_bytes", C.c_int),
                ("gpu_cache", C.c_void_p), ("segment_group", C.c_void_p), ("segment_size", C.c_int)]


MB_CACHE_LRU, MB_CACHE_LFU, MB_CACHE_WEIGHT = 0, 1, 2


class MbSegcacheStats(C.Structure):
    _fields_ = [(k, C.c_ulonglong) for k in ("hits", "misses", "admissions", "evictions", "bytes_h2d", "resident")]


class MbOffsetGPU(C.Structure):
    _fields_ = [("lo_off", C.c_void_p)] + [(f"dim_off{i}", C.c_void_p) for i in range(1, 5)]


MB_MLP_IN, MB_MLP_HIDDEN, MB_MLP_OUT, MB_MLP_PARAMS = 24, 64, 2, 5890
F32 = C.c_float

class MbCostPipeline(C.Structure):
    _fields_ = [("num_filters", C.c_int), ("filter_sel", C.c_double * MB_MAX_FILTERS), ("num_probes", C.c_int),
                ("probe_sel", C.c_double * MB_MAX_PROBES), ("group_by", C.c_int), ("num_aggr", C.c_int)]


SIGNATURES.update({
    "mb_cost_calculate": (C.c_double, [PS(MbCostPipeline), PS(C.c_int), C.c_double]),
    "mb_cost_cpu_ms": (C.c_double, [PS(MbCostPipeline), C.c_double]),
    "mb_cost_transfer_ms": (C.c_double, [C.c_double, C.c_int]),
    "mb_place_segments": (I, [I, P, P, C.c_double, C.c_double, P, P]),
    "mb_cost_build_ms": (C.c_double, [C.c_double]),
    "mb_cost_segments": (I, [PS(MbCostPipeline), I, P, P, P, P, P]),
    "mb_mlp_forward": (I, [P, P, I, P, P]),
    "mb_mlp_backward": (I, [P, P, P, I, P, P, P]),
    "mb_mlp_adam": (I, [P, P, P, P, I, F32, F32, F32, F32, I, F32, P]),
    "mb_star_select": (I, [PS(MbStarArgs), P, I64, P, P, I64, P, P]),
    "mb_filter_GPU2": (I, [P, PS(MbFilterArgsGPU), PS(MbOffsetGPU), I, P, I, P, P]),
    "mb_filter_probe_GPU2": (I, [P, PS(MbFilterArgsGPU), PS(MbProbeArgsGPU), PS(MbOffsetGPU), I, P, I, P, P]),
    "mb_probe_GPU2": (I, [P, PS(MbProbeArgsGPU), PS(MbOffsetGPU), I, P, I, P, P]),
    "mb_filter_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbFilterArgsGPU), PS(MbOffsetGPU), I, P, P]),
    "mb_filter_probe_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbFilterArgsGPU), PS(MbProbeArgsGPU), PS(MbOffsetGPU), I, P,
                                 P]),
    "mb_probe_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbProbeArgsGPU), PS(MbOffsetGPU), I, P, P]),
    "mb_filter_probe_group_by_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbFilterArgsGPU), PS(MbProbeArgsGPU),
                                          PS(MbGroupbyArgsGPU), I, P, P]),
    "mb_probe_group_by_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbProbeArgsGPU), PS(MbGroupbyArgsGPU), I, P, P]),
    "mb_groupByGPU": (I, [P, PS(MbOffsetGPU), PS(MbGroupbyArgsGPU), I, P, P]),
    "mb_aggregationGPU": (I, [P, P, PS(MbGroupbyArgsGPU), I, P, P]),
    "mb_probe_aggr_GPU2": (I, [P, PS(MbProbeArgsGPU), PS(MbGroupbyArgsGPU), I, P, I, P, P]),
    "mb_probe_aggr_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbProbeArgsGPU), PS(MbGroupbyArgsGPU), I, P, P]),
    "mb_filter_probe_aggr_GPU3": (I, [P, PS(MbOffsetGPU), PS(MbFilterArgsGPU), PS(MbProbeArgsGPU),
                                      PS(MbGroupbyArgsGPU), I, P, P]),
    "mb_build_GPU3": (I, [P, P, PS(MbFilterArgsGPU), PS(MbBuildArgsGPU), I, P, P]),
    "mb_build_GPU_minmax": (I, [P, PS(MbFilterArgsGPU), PS(MbBuildArgsGPU), I, P, P, P, I, P, P]),
    "mb_build_GPU_minmax2": (I, [P, P, PS(MbFilterArgsGPU), PS(MbBuildArgsGPU), I, P, P, P, P]),
    "mb_segcache_create": (P, [I, I64, I, I, I, I]),
    "mb_segcache_destroy": (None, [P]),
    "mb_segcache_pool": (P, [P]),
    "mb_segcache_slot": (I, [P, I, I]),
    "mb_segcache_col_idx": (I, [P, I, P]),
    "mb_segcache_begin_query": (None, [P]),
    "mb_segcache_touch": (I, [P, I, I]),
    "mb_segcache_set_weight": (I, [P, I, I, C.c_double]),
    "mb_segcache_admit": (I, [P, I, I, P, I, P, PS(I)]),
    "mb_segcache_evict": (I, [P, I, I]),
    "mb_segcache_admit_segments": (I, [P, P, I, P, I, P, P, P, PS(I), PS(C.c_ulonglong)]),
    "mb_segcache_replace": (I, [P, P, P, P, P]),
    "mb_segcache_get_stats": (I, [P, PS(MbSegcacheStats)]),
    "mb_segcache_reserve": (I, [P, I64, PS(C.c_int64)]),
    "mb_segcache_stage": (I, [P, I64, P, I, P]),
    "mb_cpu_threads": (I, []),
    "mb_cpu_build_pht": (I, [P, I, I, I, P, P, I, P, I, I, I, I, PS(C.c_uint)]),
    "mb_cpu_star_query": (I, [PS(MbStarArgs), P, I64, I, PS(C.c_uint)]),
    "mb_cpu_star_select": (I, [PS(MbStarArgs), P, I64, P, P, I64, PS(C.c_int64), I, PS(C.c_uint)]),
    "mb_pat_build": (I, [P, I, I, I, P, I, P, I, P, I, P, P]),
    "mb_batch_workspace_bytes": (C.c_size_t, [PS(MbBatchArgs)]),
    "mb_batch_run": (I, [PS(MbBatchArgs), P]),
})
