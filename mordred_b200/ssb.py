"""Star-schema queries on the C ABI: synthetic tables and the three query templates.

* filter-aggregate — the q11 form (src/ssb/q11.cu:25-93): SUM(extendedprice*discount)
  over orderdate in [19930101, 19931231], discount in [1, 3], quantity < 25.
* Query A — the q21 form (src/ssb/q21.cu): part.category = c, supplier.region = r,
  probe supplier -> part(brand) -> date(year), SUM(revenue) grouped by (year, brand).
* Query B — the q41 form (src/ssb/q41.cu): customer.region, supplier.region,
  part.mfgr in {m1, m2}, probe supplier -> customer(nation) -> part -> date(year),
  SUM(revenue - supplycost) grouped by (year, c_nation).

Device memory, streams and pinned host buffers come from PyTorch; every kernel is
the library's. The date table spans 1992-01-01..1998-12-31 (2,557 days), so its hash
table has 19981231 - 19920101 + 1 = 61,131 slots; the reference's 61,130
(src/ssb/q21.cu:152) would wrap 19981231 onto 19920101's slot.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L

DATE_MIN = 19920101
DATE_SLOTS = 19981231 - 19920101 + 1          # 61,131
REFERENCE_DATE_SLOTS = 19981230 - 19920101 + 1  # 61,130 as in the reference
QA_GROUPS = (1998 - 1992 + 1) * (5 * 5 * 40)    # 7,000
QB_GROUPS = (1998 - 1992 + 1) * 25              # 175

FACT_COLUMNS = {
    "lo_orderdate": L.MB_LO_ORDERDATE, "lo_quantity": L.MB_LO_QUANTITY,
    "lo_discount": L.MB_LO_DISCOUNT, "lo_extendedprice": L.MB_LO_EXTENDEDPRICE,
    "lo_suppkey": L.MB_LO_SUPPKEY, "lo_custkey": L.MB_LO_CUSTKEY,
    "lo_partkey": L.MB_LO_PARTKEY, "lo_revenue": L.MB_LO_REVENUE,
    "lo_supplycost": L.MB_LO_SUPPLYCOST,
}
DIM_COLUMNS = {
    "d_datekey": L.MB_D_DATEKEY, "d_year": L.MB_D_YEAR, "d_yearmonthnum": L.MB_D_YEARMONTHNUM,
    "s_suppkey": L.MB_S_SUPPKEY, "s_city": L.MB_S_CITY, "s_nation": L.MB_S_NATION,
    "s_region": L.MB_S_REGION, "c_custkey": L.MB_C_CUSTKEY, "c_city": L.MB_C_CITY,
    "c_nation": L.MB_C_NATION, "c_region": L.MB_C_REGION, "p_partkey": L.MB_P_PARTKEY,
    "p_brand1": L.MB_P_BRAND1, "p_category": L.MB_P_CATEGORY, "p_mfgr": L.MB_P_MFGR,
}

Q11_COLUMNS = ["lo_orderdate", "lo_discount", "lo_quantity", "lo_extendedprice"]
QA_FACT = ["lo_suppkey", "lo_partkey", "lo_orderdate", "lo_revenue"]
QB_FACT = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost"]
QA_DIMS = ["d_datekey", "d_year", "s_suppkey", "s_region", "p_partkey", "p_brand1", "p_category"]
QB_DIMS = ["d_datekey", "d_year", "s_suppkey", "s_region", "c_custkey", "c_region", "c_nation",
           "p_partkey", "p_mfgr"]


@dataclass
class Sizes:
    lo_len: int
    s_len: int = 40_000
    c_len: int = 600_000
    p_len: int = 1_000_000
    d_len: int = 2_557

    def dim_len(self, name: str) -> int:
        return {"d": self.d_len, "s": self.s_len, "c": self.c_len, "p": self.p_len}[name[0]]


def _stream(stream=None) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _p(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


# ---- synthetic tables ----------------------------------------------------------------

def gen_device(sizes: Sizes, seed: int, fact: list[str], dims: list[str], device="cuda",
               stream=None) -> dict[str, torch.Tensor]:
    """Generate the named columns on the GPU with the library's seeded generator."""
    out: dict[str, torch.Tensor] = {}
    s = _stream(stream)
    for name in fact:
        t = torch.empty(sizes.lo_len, dtype=torch.int32, device=device)
        L.call("mb_gen_fact_column", FACT_COLUMNS[name], seed, 0, sizes.lo_len, sizes.s_len,
               sizes.c_len, sizes.p_len, _p(t), s)
        out[name] = t
    for name in dims:
        n = sizes.dim_len(name)
        t = torch.empty(n, dtype=torch.int32, device=device)
        L.call("mb_gen_dim_column", DIM_COLUMNS[name], seed, n, _p(t), s)
        out[name] = t
    return out


def gen_host(sizes: Sizes, seed: int, fact: list[str], dims: list[str], nthreads: int = 0,
             pinned: bool = False) -> dict[str, np.ndarray]:
    """Generate the named columns on the host (bit-identical to :func:`gen_device`)."""
    out: dict[str, np.ndarray] = {}
    for name in fact:
        if pinned:
            t = torch.empty(sizes.lo_len, dtype=torch.int32, pin_memory=True)
            a = t.numpy()
        else:
            a = np.empty(sizes.lo_len, dtype=np.int32)
        L.call("mb_gen_fact_column_host", FACT_COLUMNS[name], seed, 0, sizes.lo_len, sizes.s_len,
               sizes.c_len, sizes.p_len, a.ctypes.data, nthreads)
        out[name] = a
    for name in dims:
        n = sizes.dim_len(name)
        a = np.empty(n, dtype=np.int32)
        L.call("mb_gen_dim_column_host", DIM_COLUMNS[name], seed, n, a.ctypes.data, nthreads)
        out[name] = a
    return out


# ---- result canonicalisation -----------------------------------------------------------

def crystal4_groups(res: np.ndarray) -> list[tuple[int, int, int]]:
    """Non-empty groups of an int[4*G] result as sorted (key0, key1, signed 64-bit sum).

    A group is non-empty when its first key (the year) is nonzero, the rule the
    reference's printers use (src/ssb/q21.cu:198-203, src/cpu/ssb/q41.cpp:168-173)."""
    r = np.ascontiguousarray(res, dtype=np.int32).reshape(-1, 4)
    sums = r[:, 2:4].copy().view(np.int64).reshape(-1)
    out = [(int(r[g, 0]), int(r[g, 1]), int(sums[g])) for g in np.nonzero(r[:, 0])[0]]
    return sorted(out)


def engine6_groups(res: np.ndarray) -> list[tuple[int, int, int, int, int]]:
    """Touched groups of an int[6*G] engine result as sorted (g1, g2, g3, g4, sum)."""
    r = np.ascontiguousarray(res, dtype=np.int32).reshape(-1, 6)
    sums = r[:, 4:6].copy().view(np.int64).reshape(-1)
    nz = np.nonzero(np.any(r[:, :4] != 0, axis=1) | (sums != 0))[0]
    return sorted((int(r[g, 0]), int(r[g, 1]), int(r[g, 2]), int(r[g, 3]), int(sums[g])) for g in nz)


def query_a_dense(res: np.ndarray) -> np.ndarray:
    """Query A as the dense [year-1992][brand] int64 array (7 x 1000)."""
    r = np.ascontiguousarray(res, dtype=np.int32).reshape(-1, 4)
    sums = r[:, 2:4].copy().view(np.int64).reshape(-1)   # index brand*7 + year-1992
    return sums.reshape(1000, 7).T.copy()


# ---- query workspace and templates ---------------------------------------------------

@dataclass
class StarWorkspace:
    """Hash tables, presence bitmaps and result buffers for Query A / Query B."""
    sizes: Sizes
    device: str = "cuda"
    date_slots: int = DATE_SLOTS
    t: dict = field(default_factory=dict)

    def __post_init__(self):
        z = lambda n: torch.zeros(n, dtype=torch.int32, device=self.device)
        s = self.sizes
        self.t = {
            "ht_s": z(s.s_len),                # MB_HT_KEY (supplier existence)
            "ht_c": z(2 * s.c_len),            # MB_HT_KEY_VAL (custkey -> nation)
            "ht_p_a": z(2 * s.p_len),          # MB_HT_KEY_VAL (partkey -> brand)
            "ht_p_b": z(s.p_len),              # MB_HT_KEY (part existence)
            "ht_d": z(2 * self.date_slots),    # MB_HT_KEY_VAL (datekey -> year)
            "res_a": z(4 * QA_GROUPS),
            "res_b": z(4 * QB_GROUPS),
            "rev": torch.zeros(1, dtype=torch.int64, device=self.device),
            "cnt": torch.zeros(1, dtype=torch.int32, device=self.device),
        }

    def __getitem__(self, k):
        return self.t[k]


def q11(t: dict, n: int, ws: StarWorkspace | None = None, stream=None, zero=True) -> torch.Tensor:
    """Filter-aggregate (src/ssb/q11.cu). Returns the device uint64 revenue (int64 tensor)."""
    rev = ws["rev"] if ws is not None else torch.zeros(1, dtype=torch.int64, device=t["lo_orderdate"].device)
    cnt = ws["cnt"] if ws is not None else torch.zeros(1, dtype=torch.int32, device=rev.device)
    if zero:
        rev.zero_()
        cnt.zero_()
    L.call("mb_q11_query", _p(t["lo_orderdate"]), _p(t["lo_discount"]), _p(t["lo_quantity"]),
           _p(t["lo_extendedprice"]), n, _p(rev), _p(cnt), _stream(stream))
    return rev


def query_a(t: dict, ws: StarWorkspace, category: int = 1, region: int = 1, stream=None) -> torch.Tensor:
    """Query A: builds (src/ssb/q21.cu:74-138) then the fused probe (q21.cu:25-72)."""
    build_a(t, ws, category, region, stream)
    return probe_a(t, ws, stream)


def build_a(t: dict, ws: StarWorkspace, category: int = 1, region: int = 1, stream=None) -> None:
    s, st = ws.sizes, _stream(stream)
    for k in ("ht_s", "ht_p_a", "ht_d", "res_a"):
        ws[k].zero_()
    L.call("mb_build_pht", _p(t["s_region"]), L.MB_FILTER_EQ, region, 0, _p(t["s_suppkey"]), None,
           s.s_len, _p(ws["ht_s"]), s.s_len, 0, None, st)
    L.call("mb_build_pht", _p(t["p_category"]), L.MB_FILTER_EQ, category, 0, _p(t["p_partkey"]),
           _p(t["p_brand1"]), s.p_len, _p(ws["ht_p_a"]), s.p_len, 0, None, st)
    L.call("mb_build_pht", None, 0, 0, 0, _p(t["d_datekey"]), _p(t["d_year"]), s.d_len,
           _p(ws["ht_d"]), ws.date_slots, DATE_MIN, None, st)


def probe_a(t: dict, ws: StarWorkspace, stream=None) -> torch.Tensor:
    s, st = ws.sizes, _stream(stream)
    L.call("mb_q21_probe", _p(t["lo_orderdate"]), _p(t["lo_partkey"]), _p(t["lo_suppkey"]),
           _p(t["lo_revenue"]), s.lo_len, _p(ws["ht_s"]), s.s_len, _p(ws["ht_p_a"]), s.p_len,
           _p(ws["ht_d"]), ws.date_slots, _p(ws["res_a"]), st)
    return ws["res_a"]


def query_b(t: dict, ws: StarWorkspace, c_region: int = 1, s_region: int = 1, mfgr=(0, 1),
            stream=None) -> torch.Tensor:
    """Query B: builds (src/ssb/q41.cu:82-167) then the fused probe (q41.cu:25-80)."""
    build_b(t, ws, c_region, s_region, mfgr, stream)
    return probe_b(t, ws, stream)


def build_b(t: dict, ws: StarWorkspace, c_region: int = 1, s_region: int = 1, mfgr=(0, 1),
            stream=None) -> None:
    s, st = ws.sizes, _stream(stream)
    for k in ("ht_s", "ht_c", "ht_p_b", "ht_d", "res_b"):
        ws[k].zero_()
    L.call("mb_build_pht", _p(t["s_region"]), L.MB_FILTER_EQ, s_region, 0, _p(t["s_suppkey"]), None,
           s.s_len, _p(ws["ht_s"]), s.s_len, 0, None, st)
    L.call("mb_build_pht", _p(t["c_region"]), L.MB_FILTER_EQ, c_region, 0, _p(t["c_custkey"]),
           _p(t["c_nation"]), s.c_len, _p(ws["ht_c"]), s.c_len, 0, None, st)
    L.call("mb_build_pht", _p(t["p_mfgr"]), L.MB_FILTER_EQ_OR_EQ, mfgr[0], mfgr[1], _p(t["p_partkey"]),
           None, s.p_len, _p(ws["ht_p_b"]), s.p_len, 0, None, st)
    L.call("mb_build_pht", None, 0, 0, 0, _p(t["d_datekey"]), _p(t["d_year"]), s.d_len,
           _p(ws["ht_d"]), ws.date_slots, DATE_MIN, None, st)


def probe_b(t: dict, ws: StarWorkspace, stream=None) -> torch.Tensor:
    s, st = ws.sizes, _stream(stream)
    L.call("mb_q41_probe", _p(t["lo_orderdate"]), _p(t["lo_partkey"]), _p(t["lo_custkey"]),
           _p(t["lo_suppkey"]), _p(t["lo_revenue"]), _p(t["lo_supplycost"]), s.lo_len,
           _p(ws["ht_p_b"]), s.p_len, _p(ws["ht_s"]), s.s_len, _p(ws["ht_c"]), s.c_len,
           _p(ws["ht_d"]), ws.date_slots, _p(ws["res_b"]), st)
    return ws["res_b"]


class HostStarRunner:
    """Query A + Query B over host-resident tables: every :meth:`run` copies the
    columns from pinned host memory to the GPU, builds, probes and copies both result
    arrays back — the end-to-end form of the workload, as an executor that receives
    host columns would run it."""

    def __init__(self, host_tables: dict, sizes: Sizes, device="cuda"):
        self.sizes = sizes
        self.host = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in host_tables.items()}
        self.dev = {k: torch.empty_like(v, device=device) for k, v in self.host.items()}
        self.ws = StarWorkspace(sizes, device=device)
        self.out_a = torch.empty(4 * QA_GROUPS, dtype=torch.int32).pin_memory()
        self.out_b = torch.empty(4 * QB_GROUPS, dtype=torch.int32).pin_memory()

    @property
    def h2d_bytes(self) -> int:
        return sum(v.numel() * v.element_size() for v in self.host.values())

    @property
    def d2h_bytes(self) -> int:
        return (self.out_a.numel() + self.out_b.numel()) * 4

    def run(self, stream=None) -> tuple[torch.Tensor, torch.Tensor]:
        for k, v in self.host.items():
            self.dev[k].copy_(v, non_blocking=True)
        ra = query_a(self.dev, self.ws, stream=stream)
        rb = query_b(self.dev, self.ws, stream=stream)
        self.out_a.copy_(ra, non_blocking=True)
        self.out_b.copy_(rb, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self.out_a, self.out_b


def star_args(**kw) -> L.MbStarArgs:
    """Build an :class:`MbStarArgs` from keyword fields (filters/probes as dict lists).
    The struct keeps a reference to every array whose address it holds, so the arrays
    live as long as the struct does."""
    a = L.MbStarArgs()
    a.count_after = -1
    filters = kw.pop("filters", [])
    probes = kw.pop("probes", [])
    aggr = kw.pop("aggr", [])
    a._keep = [filters, probes, aggr, dict(kw)]
    a.num_filters = len(filters)
    for i, f in enumerate(filters):
        a.filter[i] = L.MbFilter(_p(f["col"]), f.get("mode", L.MB_FILTER_BETWEEN), f["c1"], f.get("c2", 0))
    a.num_probes = len(probes)
    for i, q in enumerate(probes):
        a.probe[i] = L.MbProbe(_p(q["fkey"]), _p(q["ht"]), q["num_slots"], q.get("key_min", 0),
                               q["layout"], q.get("min_val", 0), q.get("unique_val", 0),
                               q.get("res_slot", -1), _p(q.get("presence")))
    for i, col in enumerate(aggr):
        a.aggr[i] = _p(col)
    for k, v in kw.items():
        if k in ("res", "count", "gpu_cache", "segment_group", "rows"):
            v = _p(v)
        setattr(a, k, v)
    return a


def star_query(args: L.MbStarArgs, stream=None) -> None:
    L.check("mb_star_query", L.lib().mb_star_query(C.byref(args), _stream(stream)))
