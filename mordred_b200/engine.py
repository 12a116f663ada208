"""Segmented execution of star queries over a host-resident fact table: segment skipping,
a GPU segment cache, CPU/GPU placement by a planner, concurrent CPU and GPU halves, and
the merge of their results.

Restates the reference's executor path for one query (src/gpudb/QueryProcessing.cu:
runQuery :1347-1471, executeTableDim :109-152, executeTableFact_v1 :201-437) on the
library's operators:

* :class:`SegmentedTable` — the fact table in pinned host memory, sorted by orderdate
  (as the reference's LINEORDERSORT files, src/gpudb/common.h:110-135) and split into
  segments of 1,048,576 rows (common.h:73), with per-segment min/max of every column
  (minmax.cpp:28-45); dimension tables on the GPU and the host.
* :class:`Executor` — per query: skip segments whose orderdate range misses the query's
  (QueryOptimizer.cu:1641-1662 checkPredicate); ask the planner for each remaining
  segment's CPU and GPU milliseconds and split them (mb_place_segments); run the GPU
  share from the segment cache (missing column segments admitted on the query's stream,
  in waves when the cache cannot hold them all at once) with one fused launch per wave,
  and concurrently the CPU share with the CPU engine over the pinned host columns; add
  the two partial results (CPUProcessing.cu:1786-1819 merge).
* :meth:`Executor.profile_segments` — per-segment timings on each device, the log the
  learned planner trains on.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import batch as B
from . import cpu, ssb
from .planner import QueryContext, analytic_ms, features, place
from .segcache import SegmentCache

SEG = 1 << 20
FACT = list(B.BATCH_FACT)                      # column id = index (the cache's column numbering)
COL_ID = {name: i for i, name in enumerate(FACT)}
NEEDED = {"agg": ["lo_orderdate", "lo_discount", "lo_quantity", "lo_extendedprice"],
          "qa": ["lo_orderdate", "lo_suppkey", "lo_partkey", "lo_revenue"],
          "qb": ["lo_orderdate", "lo_suppkey", "lo_custkey", "lo_partkey", "lo_revenue", "lo_supplycost"]}
DIMS = ["d_datekey", "d_year", "s_suppkey", "s_region", "c_custkey", "c_region", "c_nation", "p_partkey", "p_mfgr",
        "p_category", "p_brand1"]
CAL = np.array(B.CALENDAR, dtype=np.int64)
DAY_OF = {d: i for i, d in enumerate(B.CALENDAR)}


def _day(date: int) -> int:
    """Index of a yyyymmdd value in the calendar (dates between calendar days round up)."""
    return int(np.searchsorted(CAL, date))


class SegmentedTable:
    """n fact rows (the batch columns) in pinned host memory, orderdate ascending: row r
    has calendar day floor(r * 2557 / n), every other column from the seeded generator."""

    def __init__(self, n_rows: int, seed: int, sizes: ssb.Sizes | None = None, device="cuda",
                 columns: list[str] | None = None):
        self.n = n_rows
        self.nseg = (n_rows + SEG - 1) // SEG
        if self.nseg > 32767:
            raise ValueError("at most 32,767 segments")
        self.seg_rows = np.full(self.nseg, SEG, np.int32)
        self.seg_rows[-1] = n_rows - (self.nseg - 1) * SEG
        self.sizes = sizes or ssb.Sizes(lo_len=n_rows)
        self.seed = seed
        self.columns = columns or FACT
        self.host_t = {}
        self.host = {}
        self.min = {}
        self.max = {}
        st = ssb._stream()
        chunk = 64 * SEG
        buf = torch.empty(chunk, dtype=torch.int32, device=device)
        cal = torch.tensor(CAL, dtype=torch.int32, device=device)
        for name in self.columns:
            h = torch.empty(n_rows, dtype=torch.int32, pin_memory=True)
            mins = np.empty(self.nseg, np.int32)
            maxs = np.empty(self.nseg, np.int32)
            for r0 in range(0, n_rows, chunk):
                cnt = min(chunk, n_rows - r0)
                if name == "lo_orderdate":
                    r = torch.arange(r0, r0 + cnt, dtype=torch.int64, device=device)
                    buf[:cnt] = cal[(r * len(CAL)) // n_rows]
                else:
                    L.call("mb_gen_fact_column", ssb.FACT_COLUMNS[name], seed, r0, cnt, self.sizes.s_len,
                           self.sizes.c_len, self.sizes.p_len, buf.data_ptr(), st)
                full = cnt // SEG
                s0 = r0 // SEG
                if full:
                    v = buf[: full * SEG].view(full, SEG)
                    mins[s0: s0 + full] = v.amin(1).cpu().numpy()
                    maxs[s0: s0 + full] = v.amax(1).cpu().numpy()
                if cnt % SEG:
                    v = buf[full * SEG: cnt]
                    mins[s0 + full], maxs[s0 + full] = int(v.min()), int(v.max())
                h[r0: r0 + cnt].copy_(buf[:cnt])
            self.host_t[name] = h
            self.host[name] = h.numpy()
            self.min[name], self.max[name] = mins, maxs
        del buf
        self.dims = ssb.gen_device(self.sizes, seed, [], DIMS)
        self.hdims = {k: v.cpu().numpy() for k, v in self.dims.items()}
        self.seg_day_lo = np.array([_day(int(x)) for x in self.min["lo_orderdate"]])
        self.seg_day_hi = np.array([_day(int(x)) for x in self.max["lo_orderdate"]])

    def ptr(self, name: str, seg: int) -> int:
        return self.host[name].ctypes.data + seg * SEG * 4


def _small_sel(q: B.Query) -> dict:
    w = lambda r, n: (r[1] - r[0] + 1) / n
    out = {"discount": 1.0, "quantity": 1.0, "s": 1.0, "c": 1.0, "p": 1.0}
    if q.template == "agg":
        out["discount"], out["quantity"] = w(q.discount, 11), w(q.quantity, 50)
    elif q.template == "qa":
        out["s"], out["p"] = w(q.s_region, 5), w(q.category, 25)
    else:
        out["s"], out["c"], out["p"] = w(q.s_region, 5), w(q.c_region, 5), w(q.mfgr, 5)
    return out


@dataclass
class QueryRun:
    """Outcome of one query: its result array (host), timings and placement."""
    result: np.ndarray
    ms: float
    candidates: int
    skipped: int
    gpu_segments: int
    cpu_segments: int
    waves: int
    predicted_makespan_ms: float
    gpu_ms: float = 0.0          # device time of the GPU share (builds, copies, launches)
    cpu_ms: float = 0.0          # wall time of the CPU share (builds, CPU engine)
    admitted: int = 0
    extra: dict = field(default_factory=dict)


def host_tables(sizes: ssb.Sizes) -> dict:
    """Zeroed host hash tables of the three query forms (the CPU share's builds)."""
    n = {"s": sizes.s_len, "c": 2 * sizes.c_len, "p_key": sizes.p_len, "p_kv": 2 * sizes.p_len,
         "d": 2 * ssb.DATE_SLOTS}
    return {k: np.zeros(v, np.int32) for k, v in n.items()}


class CpuShare:
    """Segment skipping, the fused pipeline's arguments and the CPU side of a query's
    segments: filtered builds of its hash tables on the host (build_CPU,
    CPUProcessing.cu:1034-1104) and the fused pipeline over a list of segments of the
    pinned host columns (CPUProcessing.cu:723-866). Needs `t` (the table) and `hht` (host
    hash tables, :func:`host_tables`)."""

    t: SegmentedTable
    hht: dict
    cpu_nthreads: int = 0  # host threads of the CPU side (0: every thread of the engine's pool)

    def candidates(self, q: B.Query) -> np.ndarray:
        """Segments whose orderdate [min, max] meets the query's range (and, for the
        filter-aggregate, whose discount and quantity ranges meet the query's)."""
        t = self.t
        ok = (t.max["lo_orderdate"] >= q.date[0]) & (t.min["lo_orderdate"] <= q.date[1])
        if q.template == "agg":
            for name, r in (("lo_discount", q.discount), ("lo_quantity", q.quantity)):
                if name in t.min:
                    ok &= (t.max[name] >= r[0]) & (t.min[name] <= r[1])
        return np.nonzero(ok)[0]

    def build_cpu(self, q: B.Query) -> None:
        if q.template == "agg":
            return
        d, s, h = self.t.hdims, self.t.sizes, self.hht
        BT = L.MB_FILTER_BETWEEN
        h["s"][:] = 0
        h["d"][:] = 0
        nt = self.cpu_nthreads
        cpu.build_pht(d["s_region"], BT, q.s_region[0], q.s_region[1], d["s_suppkey"], None, h["s"], s.s_len, 0,
                      L.MB_HT_KEY, nt)
        cpu.build_pht(None, 0, 0, 0, d["d_datekey"], d["d_year"], h["d"], ssb.DATE_SLOTS, ssb.DATE_MIN,
                      L.MB_HT_KEY_VAL, nt)
        if q.template == "qa":
            h["p_kv"][:] = 0
            cpu.build_pht(d["p_category"], BT, q.category[0], q.category[1], d["p_partkey"], d["p_brand1"], h["p_kv"],
                          s.p_len, 0, L.MB_HT_KEY_VAL, nt)
        else:
            h["c"][:] = 0
            h["p_key"][:] = 0
            cpu.build_pht(d["c_region"], BT, q.c_region[0], q.c_region[1], d["c_custkey"], d["c_nation"], h["c"],
                          s.c_len, 0, L.MB_HT_KEY_VAL, nt)
            cpu.build_pht(d["p_mfgr"], BT, q.mfgr[0], q.mfgr[1], d["p_partkey"], None, h["p_key"], s.p_len, 0,
                          L.MB_HT_KEY, nt)

    def args(self, q: B.Query, col, ht: dict, n_rows: int, res, **extra) -> L.MbStarArgs:
        """mb_star_args of query q; col(name) gives a column (pointer or array), ht the tables."""
        s = self.t.sizes
        BT = L.MB_FILTER_BETWEEN
        date = dict(col=col("lo_orderdate"), mode=BT, c1=q.date[0], c2=q.date[1])
        d_probe = dict(fkey=col("lo_orderdate"), ht=ht["d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                       layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)
        s_probe = dict(fkey=col("lo_suppkey"), ht=ht["s"], num_slots=s.s_len, layout=L.MB_HT_KEY)
        if q.template == "agg":
            return ssb.star_args(num_rows=n_rows, filters=[
                date, dict(col=col("lo_discount"), mode=BT, c1=q.discount[0], c2=q.discount[1]),
                dict(col=col("lo_quantity"), mode=BT, c1=q.quantity[0], c2=q.quantity[1])],
                aggr=[col("lo_extendedprice"), col("lo_discount")], agg_op=L.MB_AGG_MUL,
                res_layout=L.MB_RES_SCALAR, res=res, **extra)
        if q.template == "qa":
            probes = [s_probe, dict(fkey=col("lo_partkey"), ht=ht["p_kv"], num_slots=s.p_len, layout=L.MB_HT_KEY_VAL,
                                    unique_val=7, res_slot=1), d_probe]
            return ssb.star_args(num_rows=n_rows, filters=[date], probes=probes, aggr=[col("lo_revenue")],
                                 agg_op=L.MB_AGG_SUM, total_val=ssb.QA_GROUPS, res_layout=L.MB_RES_CRYSTAL4, res=res,
                                 **extra)
        probes = [s_probe, dict(fkey=col("lo_custkey"), ht=ht["c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL,
                                unique_val=7, res_slot=1),
                  dict(fkey=col("lo_partkey"), ht=ht["p_key"], num_slots=s.p_len, layout=L.MB_HT_KEY), d_probe]
        return ssb.star_args(num_rows=n_rows, filters=[date], probes=probes,
                             aggr=[col("lo_revenue"), col("lo_supplycost")], agg_op=L.MB_AGG_SUB,
                             total_val=ssb.QB_GROUPS, res_layout=L.MB_RES_CRYSTAL4, res=res, **extra)

    @staticmethod
    def _order(segs: np.ndarray, t: SegmentedTable) -> np.ndarray:
        """A segment list with the table's partial last segment (if listed) at the end."""
        segs = np.asarray(segs, np.int64)
        last = t.nseg - 1
        if t.seg_rows[last] != SEG and (segs == last).any():
            segs = np.concatenate([segs[segs != last], [last]])
        return segs

    def _rows(self, segs: np.ndarray) -> int:
        return int(self.t.seg_rows[segs].sum())

    def _cpu_segments(self, q: B.Query, csegs: list[int], res: np.ndarray) -> None:
        segs = self._order(np.array(csegs), self.t)
        group = segs.astype(np.int16)  # the arguments hold its address: keep it alive through the call
        a = self.args(q, lambda name: self.t.host[name], self.hht, self._rows(segs), res, segment_group=group,
                      segment_size=SEG)
        cpu.star_query(a, nthreads=self.cpu_nthreads)

    def residency(self) -> tuple[dict, float]:
        """The cache's residency as context() reads it — per column, the slot of every
        segment (< 0: not resident) — and its free share: one snapshot for the many
        contexts a window plans at once."""
        idx = {c: self.cache.col_idx(COL_ID[c]) for c in FACT}
        return idx, 1.0 - self.cache.stats()["resident"] / self.cache.num_slots

    def context(self, q: B.Query, segs: np.ndarray, snapshot: tuple | None = None) -> QueryContext:
        """The planners' view of q over `segs`: rows, in-range share of each segment's
        rows (the table is date-sorted, so a segment's dates are contiguous), residency of
        the needed columns, hash-table sizes. Needs `cache` and `cpu_threads` too;
        `snapshot` (from residency()) saves reading the cache for every query."""
        t = self.t
        segs = np.asarray(segs, np.int64)
        lo, hi = t.seg_day_lo[segs], t.seg_day_hi[segs]
        qlo, qhi = _day(q.date[0]), _day(q.date[1] + 1) - 1
        inter = np.maximum(0, np.minimum(hi, qhi) - np.maximum(lo, qlo) + 1)
        date_sel = inter / np.maximum(1, hi - lo + 1)
        need = NEEDED[q.template]
        res = np.zeros(len(segs), np.int32)
        for c in need:
            idx = snapshot[0][c] if snapshot is not None else self.cache.col_idx(COL_ID[c])
            res += idx[segs] >= 0
        s = t.sizes
        ht_bytes = {"agg": 0, "qa": 4 * (s.s_len + 2 * s.p_len + 2 * ssb.DATE_SLOTS),
                    "qb": 4 * (s.s_len + 2 * s.c_len + s.p_len + 2 * ssb.DATE_SLOTS)}[q.template]
        dim_rows = {"agg": 0, "qa": s.s_len + s.p_len + s.d_len, "qb": s.s_len + s.c_len + s.p_len + s.d_len}
        free = snapshot[1] if snapshot is not None else 1.0 - self.cache.stats()["resident"] / self.cache.num_slots
        return QueryContext(q.template, t.seg_rows[segs].astype(np.float64), date_sel.astype(np.float64),
                            _small_sel(q), len(need), res, ht_bytes, dim_rows[q.template], q.groups,
                            self.cpu_threads, free)


class Executor(CpuShare):
    def __init__(self, table: SegmentedTable, cache_slots: int = 2048, policy: str = "lru", device: int = 0,
                 max_waves: int = 16):
        self.t = table
        self.cache = SegmentCache(cache_slots, SEG, len(FACT), table.nseg, policy, device)
        s = table.sizes
        z = lambda n: torch.zeros(n, dtype=torch.int32, device="cuda")
        self.ht = {"s": z(s.s_len), "c": z(2 * s.c_len), "p_key": z(s.p_len), "p_kv": z(2 * s.p_len),
                   "d": z(2 * ssb.DATE_SLOTS)}
        self.hht = host_tables(s)
        self.max_waves = max_waves
        self.col_idx_h = torch.empty(max_waves, len(FACT), table.nseg, dtype=torch.int32, pin_memory=True)
        self.col_idx_d = torch.empty(max_waves, len(FACT), table.nseg, dtype=torch.int32, device="cuda")
        self.seg_h = torch.empty(max_waves, table.nseg, dtype=torch.int16, pin_memory=True)
        self.seg_d = torch.empty(max_waves, table.nseg, dtype=torch.int16, device="cuda")
        self.res_d = torch.zeros(4 * ssb.QA_GROUPS, dtype=torch.int32, device="cuda")
        self.res_h = torch.empty(4 * ssb.QA_GROUPS, dtype=torch.int32, pin_memory=True)
        self.cpu_threads = cpu.threads()
        self._host_ptrs = [table.ptr(c, 0) if c in table.host else None for c in FACT]
        self._ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    # ---- builds ------------------------------------------------------------------------
    def build_gpu(self, q: B.Query) -> None:
        if q.template == "agg":
            return
        d, s, st = self.t.dims, self.t.sizes, ssb._stream()
        BT = L.MB_FILTER_BETWEEN
        self.ht["s"].zero_()
        self.ht["d"].zero_()
        L.call("mb_build_pht", ssb._p(d["s_region"]), BT, q.s_region[0], q.s_region[1], ssb._p(d["s_suppkey"]), None,
               s.s_len, ssb._p(self.ht["s"]), s.s_len, 0, None, st)
        L.call("mb_build_pht", None, 0, 0, 0, ssb._p(d["d_datekey"]), ssb._p(d["d_year"]), s.d_len,
               ssb._p(self.ht["d"]), ssb.DATE_SLOTS, ssb.DATE_MIN, None, st)
        if q.template == "qa":
            self.ht["p_kv"].zero_()
            L.call("mb_build_pht", ssb._p(d["p_category"]), BT, q.category[0], q.category[1], ssb._p(d["p_partkey"]),
                   ssb._p(d["p_brand1"]), s.p_len, ssb._p(self.ht["p_kv"]), s.p_len, 0, None, st)
        else:
            self.ht["c"].zero_()
            self.ht["p_key"].zero_()
            L.call("mb_build_pht", ssb._p(d["c_region"]), BT, q.c_region[0], q.c_region[1], ssb._p(d["c_custkey"]),
                   ssb._p(d["c_nation"]), s.c_len, ssb._p(self.ht["c"]), s.c_len, 0, None, st)
            L.call("mb_build_pht", ssb._p(d["p_mfgr"]), BT, q.mfgr[0], q.mfgr[1], ssb._p(d["p_partkey"]), None,
                   s.p_len, ssb._p(self.ht["p_key"]), s.p_len, 0, None, st)

    def _launch_wave(self, q: B.Query, segs: list[int], w: int) -> None:
        segs = self._order(np.array(segs), self.t)
        for c in range(len(FACT)):
            L.call("mb_segcache_col_idx", self.cache.h, c, self.col_idx_h[w, c].data_ptr())
        self.seg_h[w, : len(segs)] = torch.from_numpy(segs.astype(np.int16))
        self.col_idx_d[w].copy_(self.col_idx_h[w], non_blocking=True)
        self.seg_d[w, : len(segs)].copy_(self.seg_h[w, : len(segs)], non_blocking=True)
        col = lambda name: self.col_idx_d[w, COL_ID[name]]
        a = self.args(q, col, self.ht, self._rows(segs), self.res_d, gpu_cache=self.cache.pool,
                      segment_group=self.seg_d[w], segment_size=SEG)
        ssb.star_query(a)

    def _admit(self, q: B.Query, segs: list[int], st: int) -> tuple[int, int]:
        """Make the query's columns of `segs` resident, in order (pinned for the running
        query); returns (segments admitted, column segments copied)."""
        cols = [COL_ID[x] for x in NEEDED[q.template]]
        return self.cache.admit_segments(cols, segs, self._host_ptrs, self.t.seg_rows, st)

    def _gpu_half(self, q: B.Query, gsegs: list[int]) -> tuple[int, int, list[int]]:
        """Enqueue the GPU share on the current stream: builds, admissions, one fused
        launch per wave. Returns (waves, column segments admitted, segments left over)."""
        st = ssb._stream()
        self.build_gpu(q)
        waves = 0
        admitted = 0
        rest = list(gsegs)
        while rest and waves < self.max_waves:
            done, copied = self._admit(q, rest, st)
            admitted += copied
            if done == 0:
                break  # not even one segment fits: the CPU takes the rest
            # launch the wave, then unpin it so the next wave may recycle its slots (copies
            # into them are ordered after its kernel on this stream)
            self._launch_wave(q, rest[:done], waves)
            waves += 1
            rest = rest[done:]
            if rest:
                self.cache.begin_query()
        return waves, admitted, rest

    def _cpu_half(self, q: B.Query, csegs: list[int], res: np.ndarray) -> None:
        self.build_cpu(q)
        self._cpu_segments(q, csegs, res)

    # ---- one query -----------------------------------------------------------------------
    def run(self, q: B.Query, planner, on_gpu: np.ndarray | None = None) -> QueryRun:
        """Run q with `planner` placing its segments (or the given placement); returns the
        merged result and timings. The CPU share runs on a second thread while this one
        enqueues the GPU share (builds, admissions, launches); the CPU also takes GPU
        segments the cache could not hold."""
        t0 = time.perf_counter()
        cand = self.candidates(q)
        self.cache.begin_query()
        span = float("nan")
        pred = {}
        if on_gpu is None:
            pc, pg, fc, fg = planner.predict(self.context(q, cand))
            on_gpu, span = place(pc, pg, fc, fg)
            pred = {"pred_gpu_ms": float(pg[on_gpu].sum() + (fg if on_gpu.any() else 0.0)),
                    "pred_cpu_ms": float(pc[~on_gpu].sum() + (fc if (~on_gpu).any() else 0.0))}
        plan_ms = (time.perf_counter() - t0) * 1e3
        gsegs = [int(s) for s in cand[on_gpu]]
        csegs = [int(s) for s in cand[~on_gpu]]
        res_len = 2 if q.template == "agg" else 4 * q.groups
        self.res_d[:res_len].zero_()
        host_res = np.zeros(res_len, np.int32)
        # the CPU share starts at once on its own thread (the library calls release the
        # interpreter lock), so it overlaps the GPU share's enqueueing as well as its work
        cpu_ms = [0.0]

        def cpu_share():
            c0 = time.perf_counter()
            self._cpu_half(q, csegs, host_res)
            cpu_ms[0] = (time.perf_counter() - c0) * 1e3

        th = threading.Thread(target=cpu_share) if csegs else None
        if th:
            th.start()
        self._ev[0].record()
        waves, admitted, left = self._gpu_half(q, gsegs) if gsegs else (0, 0, [])
        self._ev[1].record()
        if th:
            th.join()
        if left:  # segments the cache could not take: the CPU runs them now
            c0 = time.perf_counter()
            if not csegs:
                self.build_cpu(q)
            self._cpu_segments(q, left, host_res)
            cpu_ms[0] += (time.perf_counter() - c0) * 1e3
            csegs = csegs + left
        out = self.res_h[:res_len]
        out.copy_(self.res_d[:res_len])  # waits for the GPU share
        res = merge(q, out.numpy().copy(), host_res)
        ms = (time.perf_counter() - t0) * 1e3
        return QueryRun(res, ms, len(cand), self.t.nseg - len(cand), len(gsegs) - len(left), len(csegs), waves,
                        span, gpu_ms=self._ev[0].elapsed_time(self._ev[1]), cpu_ms=cpu_ms[0], admitted=admitted,
                        extra=dict(pred, plan_ms=plan_ms))

    # ---- per-segment timing logs ------------------------------------------------------------
    def profile_segments(self, q: B.Query, segs: np.ndarray) -> tuple[list[dict], dict]:
        """Per-segment costs of q on each device, as the planner should see them.

        Each listed segment runs alone on each device (CUDA events around its column
        admissions and around one fused launch over it; wall clock around the CPU engine
        over it); then all of them run together in one launch and one CPU call. A
        segment's logged cost is its share of the batched time (in proportion to its
        solo time) plus, on the GPU, its own admission copies: the marginal cost it adds
        to a query's share, without the per-call overheads a solo run pays. Features come
        from the cache state before the segment's admission. Also returns the query's
        fixed costs: hash-table builds on each device."""
        st = ssb._stream()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record()
        self.build_gpu(q)
        e[1].record()
        e[1].synchronize()
        gpu_build = e[0].elapsed_time(e[1])
        c0 = time.perf_counter()
        self.build_cpu(q)
        cpu_build = (time.perf_counter() - c0) * 1e3
        res_len = 2 if q.template == "agg" else 4 * q.groups
        host_res = np.zeros(res_len, np.int32)
        self.cache.begin_query()
        segs = [int(x) for x in segs]
        # keep the partial last segment, if listed, for the end (segment lists put it last)
        segs = [int(x) for x in self._order(np.array(segs), self.t)]
        ctx = self.context(q, np.array(segs))
        feats = features(ctx)
        a_cpu, a_gpu = analytic_ms(ctx)
        xfer, ksolo, csolo, ok = [], [], [], []
        for sg in segs:
            e[0].record()
            done, _ = self._admit(q, [sg], st)
            e[1].record()
            if done == 0:
                ok.append(False)
                xfer.append(0.0), ksolo.append(0.0), csolo.append(0.0)
                continue
            self._launch_wave(q, [sg], 0)
            e[2].record()
            e[2].synchronize()
            xfer.append(e[0].elapsed_time(e[1]))
            ksolo.append(e[1].elapsed_time(e[2]))
            c0 = time.perf_counter()
            self._cpu_segments(q, [sg], host_res)
            csolo.append((time.perf_counter() - c0) * 1e3)
            ok.append(True)
        okseg = [sg for sg, k in zip(segs, ok) if k]
        if not okseg:
            return [], {"template": q.template, "cpu_build_ms": cpu_build, "gpu_build_ms": gpu_build}
        e[0].record()
        self._launch_wave(q, okseg, 1)
        e[1].record()
        e[1].synchronize()
        kbatch = e[0].elapsed_time(e[1])
        c0 = time.perf_counter()
        self._cpu_segments(q, okseg, host_res)
        cbatch = (time.perf_counter() - c0) * 1e3
        ks = sum(k for k, o in zip(ksolo, ok) if o)
        cs = sum(c for c, o in zip(csolo, ok) if o)
        out = []
        for i, sg in enumerate(segs):
            if not ok[i]:
                continue
            out.append({"features": feats[i], "cpu_ms": cbatch * csolo[i] / cs,
                        "gpu_ms": xfer[i] + kbatch * ksolo[i] / ks, "cpu_solo_ms": csolo[i],
                        "gpu_solo_ms": xfer[i] + ksolo[i], "analytic_cpu_ms": float(a_cpu[i]),
                        "analytic_gpu_ms": float(a_gpu[i]), "template": q.template, "segment": sg,
                        "resident_frac": float(ctx.resident_cols[i]) / ctx.needed_cols})
        return out, {"template": q.template, "cpu_build_ms": cpu_build, "gpu_build_ms": gpu_build,
                     "segments": len(okseg), "gpu_batch_kernel_ms": kbatch, "cpu_batch_ms": cbatch}

def merge(q: B.Query, gpu: np.ndarray, cpu_res: np.ndarray) -> np.ndarray:
    """Add the CPU share's result into the GPU share's (src/gpudb/CPUProcessing.cu:
    1786-1819): group keys from whichever side saw the group (the year key, >= 1992,
    marks a group as seen), 64-bit sums added."""
    if q.template == "agg":
        return (gpu.view(np.uint64) + cpu_res.view(np.uint64)).view(np.int32)
    g = gpu.reshape(-1, 4).copy()
    c = cpu_res.reshape(-1, 4)
    seen = c[:, 0] != 0
    g[seen, :2] = c[seen, :2]
    sums = g[:, 2:4].copy().view(np.uint64).reshape(-1) + c[:, 2:4].copy().view(np.uint64).reshape(-1)
    g[:, 2:4] = sums.view(np.int32).reshape(-1, 2)
    return g.reshape(-1)
