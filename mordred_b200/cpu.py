"""The CPU operators of the library (host columns, host hash tables): the CPU half of
CPU/GPU split execution. Thin wrappers over ``mb_cpu_build_pht`` / ``mb_cpu_star_query``
in ``include/mordred_b200.h``; the arguments are the same :class:`MbStarArgs` the GPU
path takes (built with :func:`mordred_b200.ssb.star_args` from numpy arrays)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .ssb import _p


def threads() -> int:
    return int(L.lib().mb_cpu_threads())


def build_pht(filter_col, mode: int, c1: int, c2: int, key: np.ndarray, val, ht: np.ndarray, num_slots: int,
              key_min: int, layout: int, nthreads: int = 0) -> int:
    """Filtered perfect-hash build into `ht` (zeroed by the caller); returns status bits."""
    st = C.c_uint(0)
    L.call("mb_cpu_build_pht", _p(filter_col), mode, c1, c2, _p(key), _p(val), len(key), _p(ht), num_slots,
           key_min, layout, nthreads, C.byref(st))
    return st.value


def star_query(args: L.MbStarArgs, rows: np.ndarray | None = None, nthreads: int = 0) -> int:
    """Run the fused pipeline over host columns (optionally only the listed virtual rows,
    an int32 offset list); results accumulate into args.res. Returns status bits."""
    st = C.c_uint(0)
    if rows is not None:
        rows = np.ascontiguousarray(rows, dtype=np.int32)
    L.call("mb_cpu_star_query", C.byref(args), _p(rows), 0 if rows is None else len(rows), nthreads, C.byref(st))
    return st.value


def star_select(args: L.MbStarArgs, rows: np.ndarray | None = None, capacity: int | None = None,
                nthreads: int = 0):
    """Rows passing the pipeline's filters and probes over host columns, in row order:
    (lo_off, [dim_off per probe], status bits) — the CPU side of a CPU-select ->
    GPU-aggregate split (the offset list the GPU3 forms take)."""
    st = C.c_uint(0)
    if rows is not None:
        rows = np.ascontiguousarray(rows, dtype=np.int32)
    n = len(rows) if rows is not None else int(args.num_rows)
    cap = n if capacity is None else capacity
    lo = np.empty(max(cap, 1), np.int32)
    dims = [np.empty(max(cap, 1), np.int32) for _ in range(args.num_probes)]
    arr = (C.c_void_p * 4)(*[d.ctypes.data for d in dims], *([None] * (4 - len(dims))))
    total = C.c_int64(0)
    L.call("mb_cpu_star_select", C.byref(args), _p(rows), 0 if rows is None else len(rows), lo.ctypes.data,
           C.cast(arr, C.c_void_p), cap, C.byref(total), nthreads, C.byref(st))
    k = min(int(total.value), cap)
    return lo[:k], [d[:k] for d in dims], st.value
