"""ctypes binding of the CPU oracle (oracle/liboracle.so) and a runner for the
reference's own CPU engine built under oracle/_ref. TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

MAX_FILTERS, MAX_PROBES = 3, 4


class OrcFilter(C.Structure):
    _fields_ = [("col", C.c_void_p), ("mode", C.c_int), ("c1", C.c_int), ("c2", C.c_int)]


class OrcProbe(C.Structure):
    _fields_ = [("fkey", C.c_void_p), ("ht", C.c_void_p), ("num_slots", C.c_int), ("key_min", C.c_int),
                ("layout", C.c_int), ("min_val", C.c_int), ("unique_val", C.c_int), ("res_slot", C.c_int)]


class OrcStarArgs(C.Structure):
    _fields_ = [("num_rows", C.c_int64), ("num_filters", C.c_int), ("filter", OrcFilter * MAX_FILTERS),
                ("num_probes", C.c_int), ("probe", OrcProbe * MAX_PROBES), ("aggr", C.c_void_p * 2),
                ("agg_op", C.c_int), ("total_val", C.c_int), ("group_bias", C.c_int),
                ("res_layout", C.c_int), ("res", C.c_void_p), ("count", C.c_void_p),
                ("count_after", C.c_int), ("segment_group", C.c_void_p), ("start_offset", C.c_int64),
                ("segment_size", C.c_int), ("rows", C.c_void_p)]


_lock = threading.Lock()
_lib = None


def build_lib() -> None:
    """Build liboracle.so (and the reference binaries where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True, capture_output=True, text=True)


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            src = os.path.join(HERE, "star_oracle.c")
            if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
                build_lib()
            l = C.CDLL(LIB)
            P, I, I64 = C.c_void_p, C.c_int, C.c_int64
            l.orc_star.restype = C.c_uint
            l.orc_star.argtypes = [C.POINTER(OrcStarArgs), I]
            l.orc_build.restype = C.c_uint
            l.orc_build.argtypes = [P, I, I, I, P, P, I64, P, I, I, I, I64, P]
            l.orc_build_rows.restype = C.c_uint
            l.orc_build_rows.argtypes = [P, I, I, I, P, P, P, I64, P, I, I, I64, P, I, I]
            l.orc_select.restype = C.c_int64
            l.orc_select.argtypes = [C.POINTER(OrcStarArgs), P, P, I64, P]
            l.orc_q11.restype = C.c_ulonglong
            l.orc_q11.argtypes = [P, P, P, P, I64, I, I, I, I, I, I]
            l.orc_q21.restype = C.c_uint
            l.orc_q21.argtypes = [P, P, P, P, I64, P, P, P, I, P, P, I, P, P, I, I, I, I, P, I]
            l.orc_q41.restype = C.c_uint
            l.orc_q41.argtypes = [P, P, P, P, P, P, I64, P, P, I, P, P, I, P, P, I, P, P, P, I, I, I, I, I, I, P, I]
            l.orc_merge.restype = None
            l.orc_merge.argtypes = [P, P, I]
            _lib = l
        return _lib


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "oracle takes contiguous numpy arrays"
    return a.ctypes.data


def q11(t: dict, n: int | None = None, nthreads: int = 0, date_lo_excl=19930000, date_hi_excl=19940000,
        disc_lo=1, disc_hi=3, qty_lt=25) -> int:
    n = len(t["lo_orderdate"]) if n is None else n
    return int(lib().orc_q11(_p(t["lo_orderdate"]), _p(t["lo_discount"]), _p(t["lo_quantity"]),
                             _p(t["lo_extendedprice"]), n, date_lo_excl, date_hi_excl, disc_lo, disc_hi,
                             qty_lt, nthreads))


def q21(t: dict, d_val_len: int, category=1, region=1, nthreads: int = 0):
    """Returns (res int32[6*7000] in the reference CPU layout, status bits)."""
    res = np.zeros(6 * 7000, dtype=np.int32)
    st = lib().orc_q21(_p(t["lo_orderdate"]), _p(t["lo_partkey"]), _p(t["lo_suppkey"]), _p(t["lo_revenue"]),
                       len(t["lo_orderdate"]), _p(t["p_partkey"]), _p(t["p_brand1"]), _p(t["p_category"]),
                       len(t["p_partkey"]), _p(t["d_datekey"]), _p(t["d_year"]), len(t["d_datekey"]),
                       _p(t["s_suppkey"]), _p(t["s_region"]), len(t["s_suppkey"]), d_val_len, category, region,
                       _p(res), nthreads)
    return res, st


def q41(t: dict, d_val_len: int, c_region=1, s_region=1, mfgr=(0, 1), nthreads: int = 0):
    """Returns (res int32[4*175]: year, c_nation, u64 sum; status bits)."""
    res = np.zeros(4 * 175, dtype=np.int32)
    st = lib().orc_q41(_p(t["lo_orderdate"]), _p(t["lo_custkey"]), _p(t["lo_partkey"]), _p(t["lo_suppkey"]),
                       _p(t["lo_revenue"]), _p(t["lo_supplycost"]), len(t["lo_orderdate"]), _p(t["d_datekey"]),
                       _p(t["d_year"]), len(t["d_datekey"]), _p(t["p_partkey"]), _p(t["p_mfgr"]),
                       len(t["p_partkey"]), _p(t["s_suppkey"]), _p(t["s_region"]), len(t["s_suppkey"]),
                       _p(t["c_custkey"]), _p(t["c_region"]), _p(t["c_nation"]), len(t["c_custkey"]),
                       d_val_len, c_region, s_region, mfgr[0], mfgr[1], _p(res), nthreads)
    return res, st


def q21_groups(res6: np.ndarray):
    """Reference CPU q21 layout int[6*G] {year, brand, u64 at +2} -> sorted (year, brand, sum)."""
    r = res6.reshape(-1, 6)
    sums = r[:, 2:4].copy().view(np.int64).reshape(-1)
    return sorted((int(r[g, 0]), int(r[g, 1]), int(sums[g])) for g in np.nonzero(r[:, 0])[0])


def build_ht(filter_col, mode, c1, c2, key, val, ht, num_slots, key_min, layout, row_base=0, presence=None) -> int:
    n = len(key)
    return int(lib().orc_build(_p(filter_col), mode, c1, c2, _p(key), _p(val), n, _p(ht), num_slots, key_min,
                               layout, row_base, _p(presence)))


def _args(num_rows, filters=(), probes=(), aggr=(), agg_op=0, total_val=1, group_bias=0, res_layout=0, res=None,
          count=None, count_after=-1, segment_group=None, start_offset=0, segment_size=0, rows=None) -> OrcStarArgs:
    a = OrcStarArgs()
    a.num_rows = num_rows
    a.num_filters = len(filters)
    for i, f in enumerate(filters):
        a.filter[i] = OrcFilter(_p(f["col"]), f.get("mode", 1), f["c1"], f.get("c2", 0))
    a.num_probes = len(probes)
    for i, q in enumerate(probes):
        a.probe[i] = OrcProbe(_p(q["fkey"]), _p(q["ht"]), q["num_slots"], q.get("key_min", 0), q["layout"],
                              q.get("min_val", 0), q.get("unique_val", 0), q.get("res_slot", -1))
    for i, col in enumerate(aggr):
        a.aggr[i] = _p(col)
    a.agg_op, a.total_val, a.group_bias, a.res_layout = agg_op, total_val, group_bias, res_layout
    a.res = _p(res)
    a.count = _p(count)
    a.count_after = count_after
    a.segment_group = _p(segment_group)
    a.start_offset = start_offset
    a.segment_size = segment_size
    a.rows = _p(rows)
    return a


LAYOUT_PASS = 3  # probe layout: payload = ht[fkey[k]] (a dimension column at a passed-through offset)


def star(num_rows, nthreads=0, **kw) -> int:
    """Run the generic pipeline; `res` (numpy, zeroed) is accumulated into. Returns status bits.
    rows (optional, int32) lists the physical rows to visit (num_rows of them)."""
    return int(lib().orc_star(C.byref(_args(num_rows, **kw)), nthreads))


def select(num_rows, capacity=None, **kw):
    """Rows passing the filters and probes, in visiting order: (lo_off, [dim_off per probe],
    count, status bits)."""
    a = _args(num_rows, **kw)
    cap = num_rows if capacity is None else capacity
    lo = np.zeros(max(cap, 1), np.int32)
    dims = [np.zeros(max(cap, 1), np.int32) for _ in range(a.num_probes)]
    arr = (C.c_void_p * 4)(*[d.ctypes.data for d in dims], *([None] * (4 - len(dims))))
    st = C.c_uint(0)
    k = int(lib().orc_select(C.byref(a), lo.ctypes.data, C.cast(arr, C.c_void_p), cap, C.byref(st)))
    n = min(k, cap)
    return lo[:n], [d[:n] for d in dims], k, int(st.value)


def build_rows(filter_col, mode, c1, c2, key, val, rows, n, ht, num_slots, key_min, row_base=0, minmax=None,
               val_min=0, val_max=0) -> int:
    """Engine build (VAL_OFF) over the listed dimension rows or rows [0, n); see orc_build_rows."""
    return int(lib().orc_build_rows(_p(filter_col), mode, c1, c2, _p(key), _p(val), _p(rows), n, _p(ht), num_slots,
                                    key_min, row_base, _p(minmax), val_min, val_max))


def merge(res_cpu: np.ndarray, res_gpu: np.ndarray, num_groups: int) -> None:
    lib().orc_merge(_p(res_cpu), _p(res_gpu), num_groups)


# ---- the reference's own CPU engine (oracle/_ref) ------------------------------------

def ref_available(q: int) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"ref_q{q}"))


def run_ref(q: int, seed: int, lo_len: int, s_len: int, c_len: int, p_len: int, d_len: int, trials: int = 1,
            threads: int = 0, timeout: float = 600.0):
    """Run oracle/_ref/ref_q{q}; returns (printed result lines, [ms per trial])."""
    env = dict(os.environ)
    if threads > 0:
        env["MB_REF_THREADS"] = str(threads)
    out = subprocess.run([os.path.join(REF_DIR, f"ref_q{q}"), str(seed), str(lo_len), str(s_len), str(c_len),
                          str(p_len), str(d_len), str(trials)], capture_output=True, text=True, env=env,
                         timeout=timeout, check=True).stdout
    lines, ms = [], []
    for ln in out.splitlines():
        if ln.startswith("{"):
            ms.append(json.loads(ln)["ms"])
        else:
            lines.append(ln)
    return lines, ms


def parse_ref_groups(lines: list[str]):
    """Group rows 'year key sum' printed by the reference (last trial's block)."""
    blocks, cur = [], []
    for ln in lines:
        if ln.startswith("Result:"):
            cur = []
        elif ln.startswith("Res Count:"):
            blocks.append(cur)
        else:
            parts = ln.split()
            if len(parts) == 3 and all(p.lstrip("-").isdigit() for p in parts):
                cur.append(tuple(int(p) for p in parts))
    last = blocks[-1] if blocks else cur
    out = []
    for y, k, s in last:
        out.append((y, k, s - (1 << 64) if s >= (1 << 63) else s))
    return sorted(out)


def parse_ref_revenue(lines: list[str]) -> list[int]:
    return [int(ln.split(":")[1]) for ln in lines if ln.startswith("Revenue:")]
