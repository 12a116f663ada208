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
