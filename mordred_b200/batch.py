"""Batched multi-query star execution: query templates, a seeded workload generator,
packed attribute tables and the runners (batched, and one query at a time).

Three templates over the star schema (each a range-predicate form of the reference's
queries, so selectivity can be dialled from 1e-5 to 0.3):

* ``agg``  — filter-aggregate (src/ssb/q11.cu): orderdate, discount and quantity ranges;
  SUM(extendedprice * discount); one group.
* ``qa``   — Query A (src/ssb/q21.cu): supplier region range, part category range,
  orderdate range; SUM(revenue) by (year, brand); 7,000 groups.
* ``qb``   — Query B (src/ssb/q41.cu): customer region, supplier region, part mfgr and
  orderdate ranges; SUM(revenue - supplycost) by (year, c_nation); 175 groups.

:func:`run_batch` runs any number of them in launches of up to 256 queries of the one
batched kernel; :func:`run_alone` runs one query through the single-query path
(filtered hash-table builds + ``mb_star_query``), the reference's way of executing
one query at a time.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import ssb

F = L.MB_FIELD
# dimension words: supplier/customer region(3) nation(5) city(8); part mfgr(3)
# category(5) brand(10); date year(16); bit 31 = row present
S_REGION, S_NATION, S_CITY = F(L.MB_COL_DIM_S, 0, 3), F(L.MB_COL_DIM_S, 3, 5), F(L.MB_COL_DIM_S, 8, 8)
C_REGION, C_NATION, C_CITY = F(L.MB_COL_DIM_C, 0, 3), F(L.MB_COL_DIM_C, 3, 5), F(L.MB_COL_DIM_C, 8, 8)
P_MFGR, P_CATEGORY, P_BRAND = F(L.MB_COL_DIM_P, 0, 3), F(L.MB_COL_DIM_P, 3, 5), F(L.MB_COL_DIM_P, 8, 10)
D_YEAR = F(L.MB_COL_DIM_D, 0, 16)
FACT = {name: F(i, 0, 32) for i, name in enumerate(
    ["lo_orderdate", "lo_quantity", "lo_discount", "lo_extendedprice", "lo_suppkey", "lo_custkey", "lo_partkey",
     "lo_revenue", "lo_supplycost"])}
DIM_S, DIM_C, DIM_P, DIM_D = 1, 2, 4, 8
BATCH_FACT = ["lo_orderdate", "lo_quantity", "lo_discount", "lo_extendedprice", "lo_suppkey", "lo_custkey",
              "lo_partkey", "lo_revenue", "lo_supplycost"]
BATCH_DIMS = ["d_datekey", "d_year", "s_suppkey", "s_region", "s_nation", "s_city", "c_custkey", "c_region",
              "c_nation", "c_city", "p_partkey", "p_mfgr", "p_category", "p_brand1"]


@dataclass
class Query:
    """One query of a template with its range constants (inclusive)."""
    template: str
    date: tuple[int, int]                 # orderdate range (yyyymmdd)
    discount: tuple[int, int] = (0, 10)
    quantity: tuple[int, int] = (1, 50)
    s_region: tuple[int, int] = (0, 4)
    c_region: tuple[int, int] = (0, 4)
    category: tuple[int, int] = (0, 24)
    mfgr: tuple[int, int] = (0, 4)
    target_selectivity: float = 1.0
    meta: dict = field(default_factory=dict)
    extra: list = field(default_factory=list)  # further (field code, lo, hi) predicates

    @property
    def groups(self) -> int:
        return {"agg": 1, "qa": ssb.QA_GROUPS, "qb": ssb.QB_GROUPS}[self.template]

    def result_buffer(self, device="cuda") -> torch.Tensor:
        if self.template == "agg":
            return torch.zeros(1, dtype=torch.int64, device=device)
        return torch.zeros(4 * self.groups, dtype=torch.int32, device=device)

    def to_c(self, res: torch.Tensor) -> L.MbBatchQuery:
        q = L.MbBatchQuery()
        preds = [(FACT["lo_orderdate"], *self.date)]
        if self.template == "agg":
            preds += [(FACT["lo_discount"], *self.discount), (FACT["lo_quantity"], *self.quantity)]
            q.dims_required = 0
            q.agg_op, q.agg_field[0], q.agg_field[1] = L.MB_AGG_MUL, FACT["lo_extendedprice"], FACT["lo_discount"]
            q.num_keys, q.total_val, q.res_layout = 0, 1, L.MB_RES_SCALAR
        elif self.template == "qa":
            preds += [(S_REGION, *self.s_region), (P_CATEGORY, *self.category)]
            q.dims_required = DIM_S | DIM_P | DIM_D
            q.agg_op, q.agg_field[0] = L.MB_AGG_SUM, FACT["lo_revenue"]
            q.num_keys = 2
            q.key_field[0], q.key_min[0], q.key_mul[0] = D_YEAR, 1992, 1
            q.key_field[1], q.key_min[1], q.key_mul[1] = P_BRAND, 0, 7
            q.total_val, q.res_layout = ssb.QA_GROUPS, L.MB_RES_CRYSTAL4
        else:
            preds += [(C_REGION, *self.c_region), (S_REGION, *self.s_region), (P_MFGR, *self.mfgr)]
            q.dims_required = DIM_S | DIM_C | DIM_P | DIM_D
            q.agg_op, q.agg_field[0], q.agg_field[1] = L.MB_AGG_SUB, FACT["lo_revenue"], FACT["lo_supplycost"]
            q.num_keys = 2
            q.key_field[0], q.key_min[0], q.key_mul[0] = D_YEAR, 1992, 1
            q.key_field[1], q.key_min[1], q.key_mul[1] = C_NATION, 0, 7
            q.total_val, q.res_layout = ssb.QB_GROUPS, L.MB_RES_CRYSTAL4
        preds += list(self.extra)
        if len(preds) > L.MB_BATCH_MAX_PREDS:
            raise ValueError(f"{len(preds)} predicates; at most {L.MB_BATCH_MAX_PREDS}")
        q.num_preds = len(preds)
        for i, (f, lo, hi) in enumerate(preds):
            q.pred_field[i], q.pred_lo[i], q.pred_hi[i] = f, lo, hi
        q.res = res.data_ptr()
        return q


# ---- workload generator --------------------------------------------------------------

def _calendar() -> list[int]:
    import datetime as dt
    d0 = dt.date(1992, 1, 1)
    return [int((d0 + dt.timedelta(days=i)).strftime("%Y%m%d")) for i in range(2557)]


CALENDAR = _calendar()


def _pick_range(rng: np.random.Generator, domain_lo: int, domain_hi: int, width: int) -> tuple[int, int]:
    n = domain_hi - domain_lo + 1
    width = max(1, min(n, width))
    start = domain_lo + int(rng.integers(0, n - width + 1))
    return start, start + width - 1


SMALL_DOMAINS = {"agg": [("discount", 0, 10), ("quantity", 1, 50)],
                 "qa": [("s_region", 0, 4), ("category", 0, 24)],
                 "qb": [("c_region", 0, 4), ("s_region", 0, 4), ("mfgr", 0, 4)]}


def generate_queries(n: int, seed: int, sel_lo: float = 1e-5, sel_hi: float = 0.3,
                     templates=("agg", "qa", "qb")) -> list[Query]:
    """n queries, templates drawn uniformly, target selectivities log-uniform in
    [sel_lo, sel_hi] (attribute values are uniform, so a range's selectivity is its
    share of the domain). The small-domain predicates take a random share of
    log(selectivity); the orderdate range (2,557 days) then makes up the rest, which
    lands the product within one day of the target whenever it is reachable."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        tpl = templates[int(rng.integers(0, len(templates)))]
        sel = math.exp(rng.uniform(math.log(sel_lo), math.log(sel_hi)))
        q = Query(template=tpl, date=(CALENDAR[0], CALENDAR[-1]), target_selectivity=sel)
        small = SMALL_DOMAINS[tpl]
        share = rng.uniform(0.0, 0.8)             # part of log(sel) carried by the small predicates
        parts = rng.dirichlet(np.ones(len(small)))
        f_small = 1.0
        for (name, lo, hi), part in zip(small, parts):
            size = hi - lo + 1
            width = max(1, min(size, int(round(size * sel ** (share * part)))))
            f_small *= width / size
            setattr(q, name, _pick_range(rng, lo, hi, width))
        days = max(1, min(2557, int(round(2557 * sel / f_small))))
        a, b = _pick_range(rng, 0, 2556, days)
        q.date = (CALENDAR[a], CALENDAR[b])
        q.meta["expected_selectivity"] = f_small * days / 2557
        out.append(q)
    return out


# ---- packed attribute tables ----------------------------------------------------------

@dataclass
class Pats:
    words: dict                       # "S","C","P","D" -> int32 tensor (uint32 words)
    slots: dict
    key_min: dict

    def c_dims(self) -> L.MbPat * 4:
        arr = (L.MbPat * 4)()
        for i, k in enumerate("SCPD"):
            arr[i] = L.MbPat(self.words[k].data_ptr(), self.slots[k], self.key_min[k])
        return arr


def build_pats(t: dict, sizes: ssb.Sizes, stream=None) -> Pats:
    st = ssb._stream(stream)
    spec = {
        "S": ("s_suppkey", sizes.s_len, 0, [("s_region", S_REGION), ("s_nation", S_NATION), ("s_city", S_CITY)]),
        "C": ("c_custkey", sizes.c_len, 0, [("c_region", C_REGION), ("c_nation", C_NATION), ("c_city", C_CITY)]),
        "P": ("p_partkey", sizes.p_len, 0, [("p_mfgr", P_MFGR), ("p_category", P_CATEGORY), ("p_brand1", P_BRAND)]),
        "D": ("d_datekey", ssb.DATE_SLOTS, ssb.DATE_MIN, [("d_year", D_YEAR)]),
    }
    words, slots, kmin = {}, {}, {}
    for k, (key, nslots, km, attrs) in spec.items():
        w = torch.zeros(nslots, dtype=torch.int32, device=t[key].device)
        args = []
        for i in range(3):
            if i < len(attrs):
                args += [ssb._p(t[attrs[i][0]]), attrs[i][1]]
            else:
                args += [None, 0]
        L.call("mb_pat_build", ssb._p(t[key]), t[key].numel(), km, nslots, *args, ssb._p(w), st)
        words[k], slots[k], kmin[k] = w, nslots, km
    return Pats(words, slots, kmin)


# ---- runners ----------------------------------------------------------------------------

class BatchPlan:
    """A batch prepared for launching: argument structs per launch of up to 256 queries
    and the device workspace their query masks need (sized once, reused by every run, so
    a run allocates nothing and can be captured in a CUDA graph)."""

    def __init__(self, t: dict, pats: Pats, queries: list[Query], results: list[torch.Tensor], n_rows: int,
                 threads=0, items=0, stages=0, smem_group_bytes=-1):
        self.launches = []
        need = 0
        for base in range(0, len(queries), L.MB_BATCH_MAX_QUERIES):
            chunk = queries[base: base + L.MB_BATCH_MAX_QUERIES]
            arr = (L.MbBatchQuery * len(chunk))(*[q.to_c(results[base + i]) for i, q in enumerate(chunk)])
            a = L.MbBatchArgs()
            a.num_rows = n_rows
            for i, name in enumerate(BATCH_FACT):
                a.fact[i] = ssb._p(t[name])
            a.dim = pats.c_dims()
            a.num_queries = len(chunk)
            a.queries = C.cast(arr, C.POINTER(L.MbBatchQuery))
            a.threads, a.items_per_thread, a.stages = threads, items, stages
            a.smem_group_bytes = smem_group_bytes
            need = max(need, int(L.lib().mb_batch_workspace_bytes(C.byref(a))))
            self.launches.append((a, arr))
        device = next(iter(t.values())).device
        self.workspace = torch.empty(max(16, need), dtype=torch.uint8, device=device)
        for a, _ in self.launches:
            a.workspace, a.workspace_bytes = self.workspace.data_ptr(), self.workspace.numel()

    def run(self, stream=None) -> None:
        st = ssb._stream(stream)
        for a, _ in self.launches:
            L.check("mb_batch_run", L.lib().mb_batch_run(C.byref(a), st))

    def set_launch(self, threads=0, items=0, stages=0, smem_group_bytes=-1) -> None:
        """Change the launch configuration of every launch (0 / -1: the defaults)."""
        for a, _ in self.launches:
            a.threads, a.items_per_thread, a.stages = threads, items, stages
            a.smem_group_bytes = smem_group_bytes

    def capture(self, zero: torch.Tensor | None = None) -> torch.cuda.CUDAGraph:
        """A CUDA graph of one run (preceded by zeroing `zero`, typically the buffer from
        :func:`result_buffers`): the host-side planning and launch argument assembly happen
        once, at capture; each replay is a handful of graph nodes."""
        self.run()  # plan and load the kernels outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            if zero is not None:
                zero.zero_()
            self.run()
        return g

    def autotune(self, configs=None, reps: int = 3) -> dict:
        """Time launch configurations on this batch with CUDA events and keep the fastest.
        Results are accumulated into while timing: zero them afterwards."""
        configs = configs or BATCH_TUNE_CONFIGS
        timings = []
        for threads, items, stages, sg in configs:
            self.set_launch(threads, items, stages, sg)
            try:
                self.run()
            except L.MbError:
                continue  # does not fit in shared memory
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                self.run()
            e1.record()
            torch.cuda.synchronize()
            timings.append((e0.elapsed_time(e1) / reps, (threads, items, stages, sg)))
        if not timings:
            raise RuntimeError("no launch configuration fits this batch")
        ms, best = min(timings)
        self.set_launch(*best)
        return {"best": dict(zip(("threads", "items", "stages", "smem_group_bytes"), best)), "ms": ms,
                "timings": [(c, t) for t, c in timings]}


# launch configurations the batch autotuner tries: consumer threads, rows per thread,
# stages, shared memory for small group arrays
BATCH_TUNE_CONFIGS = [(t, i, st, sg) for t, i in ((768, 1), (960, 1), (512, 2), (256, 4))
                      for st in (2, 3) for sg in (65536, 131072)]


def result_buffers(queries: list[Query], device="cuda") -> tuple[torch.Tensor, list[torch.Tensor]]:
    """One zeroed buffer holding every query's result (so one memset clears a batch), and
    per-query views of it shaped like :meth:`Query.result_buffer`."""
    sizes = [8 if q.template == "agg" else 16 * q.groups for q in queries]
    flat = torch.zeros(sum(sizes), dtype=torch.uint8, device=device)
    views, off = [], 0
    for q, nb in zip(queries, sizes):
        v = flat[off: off + nb]
        views.append(v.view(torch.int64) if q.template == "agg" else v.view(torch.int32))
        off += nb
    return flat, views


def run_batch(t: dict, pats: Pats, queries: list[Query], results: list[torch.Tensor], n_rows: int,
              stream=None, threads=0, items=0, stages=0, smem_group_bytes=-1) -> None:
    """All queries through the batched kernel (launches of up to 256 queries)."""
    BatchPlan(t, pats, queries, results, n_rows, threads, items, stages, smem_group_bytes).run(stream)


class AloneWorkspace:
    """Per-query filtered hash tables for running queries one at a time."""

    def __init__(self, sizes: ssb.Sizes, device="cuda"):
        z = lambda n: torch.zeros(n, dtype=torch.int32, device=device)
        self.sizes = sizes
        self.ht_s, self.ht_c, self.ht_p = z(sizes.s_len), z(2 * sizes.c_len), z(2 * sizes.p_len)
        self.ht_pk, self.ht_d = z(sizes.p_len), z(2 * ssb.DATE_SLOTS)


def run_alone(t: dict, ws: AloneWorkspace, q: Query, res: torch.Tensor, n_rows: int, stream=None) -> None:
    """One query the reference's way: filtered PHT builds, then the fused probe."""
    s, st = ws.sizes, ssb._stream(stream)
    B = L.MB_FILTER_BETWEEN
    date = dict(col=t["lo_orderdate"], mode=B, c1=q.date[0], c2=q.date[1])
    if q.template == "agg":
        args = ssb.star_args(num_rows=n_rows, filters=[date, dict(col=t["lo_discount"], mode=B, c1=q.discount[0],
                                                                  c2=q.discount[1]),
                                                       dict(col=t["lo_quantity"], mode=B, c1=q.quantity[0],
                                                            c2=q.quantity[1])],
                             aggr=[t["lo_extendedprice"], t["lo_discount"]], agg_op=L.MB_AGG_MUL,
                             res_layout=L.MB_RES_SCALAR, res=res)
        ssb.star_query(args, stream)
        return
    ws.ht_s.zero_()
    ws.ht_d.zero_()
    L.call("mb_build_pht", ssb._p(t["s_region"]), B, q.s_region[0], q.s_region[1], ssb._p(t["s_suppkey"]), None,
           s.s_len, ssb._p(ws.ht_s), s.s_len, 0, None, st)
    L.call("mb_build_pht", None, 0, 0, 0, ssb._p(t["d_datekey"]), ssb._p(t["d_year"]), s.d_len, ssb._p(ws.ht_d),
           ssb.DATE_SLOTS, ssb.DATE_MIN, None, st)
    d_probe = dict(fkey=t["lo_orderdate"], ht=ws.ht_d, num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                   layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)
    s_probe = dict(fkey=t["lo_suppkey"], ht=ws.ht_s, num_slots=s.s_len, layout=L.MB_HT_KEY)
    if q.template == "qa":
        ws.ht_p.zero_()
        L.call("mb_build_pht", ssb._p(t["p_category"]), B, q.category[0], q.category[1], ssb._p(t["p_partkey"]),
               ssb._p(t["p_brand1"]), s.p_len, ssb._p(ws.ht_p), s.p_len, 0, None, st)
        probes = [s_probe, dict(fkey=t["lo_partkey"], ht=ws.ht_p, num_slots=s.p_len, layout=L.MB_HT_KEY_VAL,
                                unique_val=7, res_slot=1), d_probe]
        args = ssb.star_args(num_rows=n_rows, filters=[date], probes=probes, aggr=[t["lo_revenue"]],
                             agg_op=L.MB_AGG_SUM, total_val=ssb.QA_GROUPS, res_layout=L.MB_RES_CRYSTAL4, res=res)
    else:
        ws.ht_c.zero_()
        ws.ht_pk.zero_()
        L.call("mb_build_pht", ssb._p(t["c_region"]), B, q.c_region[0], q.c_region[1], ssb._p(t["c_custkey"]),
               ssb._p(t["c_nation"]), s.c_len, ssb._p(ws.ht_c), s.c_len, 0, None, st)
        L.call("mb_build_pht", ssb._p(t["p_mfgr"]), B, q.mfgr[0], q.mfgr[1], ssb._p(t["p_partkey"]), None, s.p_len,
               ssb._p(ws.ht_pk), s.p_len, 0, None, st)
        probes = [s_probe, dict(fkey=t["lo_custkey"], ht=ws.ht_c, num_slots=s.c_len, layout=L.MB_HT_KEY_VAL,
                                unique_val=7, res_slot=1),
                  dict(fkey=t["lo_partkey"], ht=ws.ht_pk, num_slots=s.p_len, layout=L.MB_HT_KEY), d_probe]
        args = ssb.star_args(num_rows=n_rows, filters=[date], probes=probes, aggr=[t["lo_revenue"],
                                                                                   t["lo_supplycost"]],
                             agg_op=L.MB_AGG_SUB, total_val=ssb.QB_GROUPS, res_layout=L.MB_RES_CRYSTAL4, res=res)
    ssb.star_query(args, stream)


def result_groups(q: Query, res) -> list:
    a = res.cpu().numpy() if isinstance(res, torch.Tensor) else res
    if q.template == "agg":
        return [int(np.asarray(a).view(np.int64)[0])]
    return ssb.crystal4_groups(a)
