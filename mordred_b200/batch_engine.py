"""Batched execution over the host-resident segmented table: a window of queued queries is
answered by shared scans, with the planner deciding which segments the GPU scans for all
of them and which the host cores run per query, and which column segments stay resident
in the GPU segment cache.

The reference runs one query at a time (src/gpudb/QueryProcessing.cu:1347-1471), placing
each query's segment groups on a device from the cost model (QueryOptimizer.cu:1674-1891)
and refilling its segment cache by benefit weights (CacheManager.cu:534-588). Here:

* candidates — per query, the segments whose orderdate range meets the query's
  (QueryOptimizer.cu:1641-1662); the window's union is what the GPU may have to scan.
* placement — the planner (learned MLP or the analytic model) predicts, per (query,
  candidate segment), CPU ms and GPU ms. A segment's GPU cost in the batch is the most
  expensive member's (the copies of its columns and the scan are shared by every query
  of the window); its CPU cost is the sum over the queries that need it, each with its
  share of that query's host hash-table builds. mb_place_segments splits the union to
  minimise the window's makespan.
* admission — every window the planner's predicted saving from residency (GPU ms with
  the segment's columns missing minus resident, per column) of each column segment the
  window reads is added into an exponentially weighted benefit, and the cache keeps the
  heaviest (mb_segcache_replace, the reference's SegmentReplacement with the model's
  weights). Segments the GPU scans that are not resident stream through reserved
  staging slots (mb_segcache_reserve / mb_segcache_stage) without evicting anything.
* execution — resident segments are scanned at once; staged segments go in waves,
  copies of wave w + 1 on a copy stream overlapping the scan of wave w on the kernel
  stream (two staging buffers); every scan is one batched launch (mb_batch_run with
  segment-cache addressing) per 256 queries. The host share runs concurrently on the
  CPU engine. Each query's GPU and CPU partial results merge by addition
  (CPUProcessing.cu:1786-1819).
Results equal each query run alone (integer sums; tests/test_batch_engine.py).
"""
from __future__ import annotations

import ctypes as C
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import batch as B
from . import cpu, ssb
from .engine import COL_ID, FACT, NEEDED, SEG, CpuShare, SegmentedTable, host_tables, merge
from .planner import place
from .segcache import SegmentCache


@dataclass
class WindowRun:
    """Outcome of one window: per-query merged results (host) and timings."""
    results: list
    ms: float
    queries: int
    union_segments: int
    gpu_segments: int
    cpu_segments: int
    staged_segments: int
    launches: int
    predicted_makespan_ms: float
    plan_ms: float = 0.0
    gpu_ms: float = 0.0
    cpu_ms: float = 0.0
    copied_column_segments: int = 0
    extra: dict = field(default_factory=dict)


class BatchExecutor(CpuShare):
    """Windows of queries over a :class:`SegmentedTable` with a GPU segment cache of
    `cache_slots` slots (the budget includes the staging slots)."""

    MAX_CHUNKS = 16  # 256-query launches a window may hold (4,096 queries)

    def __init__(self, table: SegmentedTable, cache_slots: int = 2048, stage_segments: int = 12, device: int = 0,
                 benefit_decay: float = 0.5):
        ncol = len(FACT)
        self.t = table
        self.cache = SegmentCache(cache_slots, SEG, ncol, table.nseg, "weight", device)
        self.stage_segments = stage_segments
        self.stage0 = self.cache.reserve(2 * stage_segments * ncol)
        self.hht = host_tables(table.sizes)
        self.cpu_threads = cpu.threads()
        dims = dict(table.dims)
        extra = [d for d in B.BATCH_DIMS if d not in dims]
        dims.update(ssb.gen_device(table.sizes, table.seed, [], extra))
        self.dims = dims
        self.pats = B.build_pats(dims, table.sizes)
        self.c_dims = self.pats.c_dims()
        self.kstream = torch.cuda.Stream()
        self.cstream = torch.cuda.Stream()
        self.max_waves = table.nseg // stage_segments + 3
        # host slot arrays per window parity: a window's copies of them may still be queued
        # behind the previous window's scans while the next window is being enqueued
        self.col_h = torch.empty(2, self.max_waves, ncol, table.nseg, dtype=torch.int32, pin_memory=True)
        self.col_d = torch.empty(self.max_waves, ncol, table.nseg, dtype=torch.int32, device="cuda")
        # per wave and query chunk (up to 256 queries a launch): the wave's segments that the
        # chunk's queries can match
        self.seg_h = torch.empty(2, self.max_waves, self.MAX_CHUNKS, table.nseg, dtype=torch.int16,
                                 pin_memory=True)
        self.seg_d = torch.empty(self.max_waves, self.MAX_CHUNKS, table.nseg, dtype=torch.int16, device="cuda")
        self._parity = 0
        self._stage_done = [None, None]  # events: the last scans that read staging buffer 0 / 1
        self._stage_buf = 0
        self._cpu_jobs: queue.Queue = queue.Queue()
        self._cpu_worker = threading.Thread(target=self._cpu_loop, daemon=True)
        self._cpu_worker.start()
        self.ws = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
        self.host_ptrs = [table.ptr(c, 0) for c in FACT]
        self.benefit = np.zeros((ncol, table.nseg))
        self.decay = benefit_decay
        self.admission = True

    # ---- planning ------------------------------------------------------------------------
    def _predict(self, planner, queries, cands):
        """Per query, the planner's (cpu_ms, gpu_ms, cpu_fixed, gpu_fixed) over its candidate
        segments, and — for admission — the predicted GPU ms each segment saves when its
        columns are resident rather than missing (batched model calls)."""
        snap = self.residency()
        ctxs = [self.context(q, c, snap) for q, c in zip(queries, cands)]
        if not self.admission:
            return planner.predict_many(ctxs), None
        lo, hi = [], []
        for ctx in ctxs:
            a = ctx.subset(slice(None))
            a.resident_cols = np.zeros_like(ctx.resident_cols)
            b = ctx.subset(slice(None))
            b.resident_cols = np.full_like(ctx.resident_cols, ctx.needed_cols)
            lo.append(a)
            hi.append(b)
        # one model call for the window's three views (as cached, all missing, all resident)
        out = planner.predict_many(ctxs + lo + hi)
        n = len(ctxs)
        base, miss, res = out[:n], out[n: 2 * n], out[2 * n:]
        saving = [np.maximum(m[1] - r[1], 0.0) for m, r in zip(miss, res)]
        return base, saving

    def _admit(self, queries, cands, saving, stream) -> int:
        """Fold this window's predicted residency savings into the benefit weights and
        replace the cache's contents by them; returns the column segments copied in."""
        win = np.zeros_like(self.benefit)
        for q, cand, sv in zip(queries, cands, saving):
            cols = [COL_ID[c] for c in NEEDED[q.template]]
            if len(cand) == 0:
                continue
            for c in cols:
                win[c, cand] += sv / len(cols)
        self.benefit = self.decay * self.benefit + win
        before = self.cache.stats()["admissions"]
        with torch.cuda.stream(stream):
            self.cache.replace(self.benefit, self.host_ptrs, self.t.seg_rows, stream.cuda_stream)
        return self.cache.stats()["admissions"] - before

    # ---- GPU share -------------------------------------------------------------------------
    def _launch(self, w: int, subsets: list, qarrs: list, cols_needed: list[int], stream) -> int:
        """One batched launch per chunk of up to 256 queries over the wave's segments that
        chunk can match (col_d[w] / seg_d[w, k] already hold the slot arrays and segment
        lists); returns launches issued."""
        launches = 0
        for k, (arr, nq, cols, _) in enumerate(qarrs):
            sub = subsets[k]
            if len(sub) == 0:
                continue
            a = L.MbBatchArgs()
            a.num_rows = self._rows(sub)
            for c in cols:
                a.fact[c] = self.col_d[w, c].data_ptr()
            a.dim = self.c_dims
            a.num_queries = nq
            a.queries = C.cast(arr, C.POINTER(L.MbBatchQuery))
            a.smem_group_bytes = -1
            a.gpu_cache = self.cache.pool
            a.segment_group = self.seg_d[w, k].data_ptr()
            a.segment_size = SEG
            need = int(L.lib().mb_batch_workspace_bytes(C.byref(a)))
            if need > self.ws.numel():
                stream.synchronize()
                self.ws = torch.empty(2 * need, dtype=torch.uint8, device="cuda")
            a.workspace, a.workspace_bytes = self.ws.data_ptr(), self.ws.numel()
            L.check("mb_batch_run", L.lib().mb_batch_run(C.byref(a), stream.cuda_stream))
            launches += 1
        return launches

    def _gpu_share(self, gsegs: np.ndarray, qarrs, cols_needed: list[int]) -> tuple[int, int, int]:
        """Scan gsegs for every query: resident segments in one launch, the others staged
        in waves; returns (launches, waves, column segments staged)."""
        ks, cs = self.kstream, self.cstream
        if len(gsegs) == 0:
            return 0, 0, 0
        idx = {c: self.cache.col_idx(c) for c in cols_needed}
        resident = np.array([all(idx[c][s] >= 0 for c in cols_needed) for s in gsegs], bool)
        waves = []
        if resident.any():
            waves.append((self._order(gsegs[resident], self.t), False))
        rest = gsegs[~resident]
        for i in range(0, len(rest), self.stage_segments):
            waves.append((self._order(rest[i: i + self.stage_segments], self.t), True))
        launches, staged = 0, 0
        done_ev = self._stage_done  # scans that last read staging buffer 0 / 1 (any window)
        buf = self._stage_buf
        col_h, seg_h = self.col_h[self._parity], self.seg_h[self._parity]
        for w, (segs, needs_stage) in enumerate(waves):
            if w >= self.max_waves:
                raise RuntimeError("more waves than the executor's slot arrays hold")
            for c in cols_needed:
                col_h[w, c, segs] = torch.from_numpy(idx[c][segs])
            if needs_stage:
                if done_ev[buf] is not None:
                    cs.wait_event(done_ev[buf])
                for j, s in enumerate(segs):
                    for c in cols_needed:
                        if idx[c][s] >= 0:
                            continue
                        slot = self.stage0 + (buf * self.stage_segments + j) * len(FACT) + c
                        self.cache.stage(slot, self.host_ptrs[c] + int(s) * SEG * 4, int(self.t.seg_rows[s]),
                                         cs.cuda_stream)
                        col_h[w, c, s] = slot
                        staged += 1
                copied = torch.cuda.Event()
                copied.record(cs)
                ks.wait_event(copied)
            subsets = [segs[mask[segs]] for _, _, _, mask in qarrs]  # keeps the partial segment last
            with torch.cuda.stream(ks):
                self.col_d[w].copy_(col_h[w], non_blocking=True)
                for k, sub in enumerate(subsets):
                    if len(sub):
                        seg_h[w, k, : len(sub)] = torch.from_numpy(sub.astype(np.int16))
                        self.seg_d[w, k, : len(sub)].copy_(seg_h[w, k, : len(sub)], non_blocking=True)
            launches += self._launch(w, subsets, qarrs, cols_needed, ks)
            if needs_stage:
                ev = torch.cuda.Event()
                ev.record(ks)
                done_ev[buf] = ev
                buf ^= 1
        self._stage_buf = buf
        return launches, len(waves), staged

    def close(self) -> None:
        """Stop the CPU worker (after the windows already handed to it)."""
        if self._cpu_worker.is_alive():
            self._cpu_jobs.put(None)
            self._cpu_worker.join(timeout=60)

    def __enter__(self) -> "BatchExecutor":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    # ---- one window ---------------------------------------------------------------------------
    def _cpu_loop(self) -> None:
        """The windows' CPU shares, one after another (they share the host hash tables)."""
        while True:
            job = self._cpu_jobs.get()
            if job is None:
                return
            fn, done, err = job
            try:
                fn()
            except BaseException as e:  # re-raised by _finish_window
                err.append(e)
            finally:
                done.set()

    def _start_window(self, queries: list[B.Query], planner) -> dict:
        """Plan a window and enqueue all of its work: admission copies, staged waves and
        scans on the device streams, its CPU share on the CPU worker. Returns what
        _finish_window needs; nothing here waits for earlier windows' device work."""
        t0 = time.perf_counter()
        ks = self.kstream
        cands = [self.candidates(q) for q in queries]
        (preds, saving) = self._predict(planner, queries, cands)
        copied = self._admit(queries, cands, saving, ks) if saving is not None else 0
        # per segment: the CPU ms of the queries that need it (each with its share of the
        # query's host builds) summed, and the most expensive member's GPU ms
        nz = [(np.asarray(c, np.int64), pc, pg, fc) for c, (pc, pg, fc, fg) in zip(cands, preds) if len(c)]
        if nz:
            seg_all = np.concatenate([c for c, _, _, _ in nz])
            cpu_all = np.concatenate([np.asarray(pc, np.float64) + fc / len(c) for c, pc, _, fc in nz])
            gpu_all = np.concatenate([np.asarray(pg, np.float64) for _, _, pg, _ in nz])
            segs, inv = np.unique(seg_all, return_inverse=True)
            cpu_cost = np.bincount(inv, weights=cpu_all, minlength=len(segs))
            gpu_cost = np.full(len(segs), -np.inf)
            np.maximum.at(gpu_cost, inv, gpu_all)
            on_gpu, span = place(cpu_cost, gpu_cost)
        else:
            segs = np.zeros(0, np.int64)
            on_gpu, span = np.zeros(0, bool), 0.0
        gsegs, csegs = segs[on_gpu], segs[~on_gpu]
        plan_ms = (time.perf_counter() - t0) * 1e3

        # result buffers (zeroed on the current stream, which the kernel stream then waits
        # for) and launch descriptors (chunks of up to 256 queries)
        flat, views = B.result_buffers(queries)
        ks.wait_stream(torch.cuda.current_stream())
        # launch chunks of up to 256 queries, grouped by the part of the date-sorted table
        # they need (queries over more than a quarter of it together, the others by their
        # first segment), so that each chunk's launch scans only the segments its queries
        # can match instead of every segment the window scans
        nseg = self.t.nseg
        order = sorted(range(len(queries)),
                       key=lambda i: (len(cands[i]) > nseg // 4, int(cands[i][0]) if len(cands[i]) else -1,
                                      len(cands[i])))
        qarrs = []
        for base in range(0, len(order), L.MB_BATCH_MAX_QUERIES):
            chunk = order[base: base + L.MB_BATCH_MAX_QUERIES]
            arr = (L.MbBatchQuery * len(chunk))(*[queries[i].to_c(views[i]) for i in chunk])
            cols = sorted({COL_ID[c] for i in chunk for c in NEEDED[queries[i].template]})
            mask = np.zeros(nseg, bool)
            for i in chunk:
                mask[cands[i]] = True
            qarrs.append((arr, len(chunk), cols, mask))
        if len(qarrs) > self.MAX_CHUNKS:
            raise ValueError(f"a window holds at most {self.MAX_CHUNKS * L.MB_BATCH_MAX_QUERIES} queries")
        cols_needed = sorted({c for _, _, cols, _ in qarrs for c in cols})

        # CPU share on the CPU worker: per query, its host tables and its CPU segments
        host_res = [np.zeros(2 if q.template == "agg" else 4 * q.groups, np.int32) for q in queries]
        on_cpu = np.zeros(self.t.nseg, bool)
        on_cpu[csegs] = True
        cpu_ms = [0.0]

        def cpu_share():
            c0 = time.perf_counter()
            for qi, (q, cand) in enumerate(zip(queries, cands)):
                mine = np.asarray(cand, np.int64)
                mine = mine[on_cpu[mine]] if len(mine) else mine
                if len(mine):
                    self.build_cpu(q)
                    self._cpu_segments(q, [int(x) for x in mine], host_res[qi])
            cpu_ms[0] = (time.perf_counter() - c0) * 1e3

        cpu_done, cpu_err = threading.Event(), []
        if len(csegs):
            self._cpu_jobs.put((cpu_share, cpu_done, cpu_err))
        else:
            cpu_done.set()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(ks)
        launches, waves, staged = self._gpu_share(gsegs, qarrs, cols_needed)
        g1.record(ks)
        self._parity ^= 1
        host = torch.empty(flat.numel(), dtype=torch.uint8, pin_memory=True)
        with torch.cuda.stream(ks):
            host.copy_(flat, non_blocking=True)
        read = torch.cuda.Event()
        read.record(ks)
        return dict(t0=t0, queries=queries, segs=segs, gsegs=gsegs, csegs=csegs, span=span, plan_ms=plan_ms,
                    copied=copied, flat=flat, qarrs=qarrs, host_res=host_res, cpu_ms=cpu_ms, cpu_done=cpu_done,
                    cpu_err=cpu_err,
                    g0=g0, g1=g1, launches=launches, waves=waves, staged=staged, host=host, read=read)

    def _finish_window(self, st: dict) -> WindowRun:
        """Wait for a started window and merge each query's GPU and CPU partial results."""
        st["cpu_done"].wait()
        st["read"].synchronize()
        if st["cpu_err"]:
            raise st["cpu_err"][0]
        done_at = time.perf_counter()
        hb = st["host"].numpy()
        results, off = [], 0
        split = len(st["csegs"]) > 0
        for q, hr in zip(st["queries"], st["host_res"]):
            nb = 8 if q.template == "agg" else 16 * q.groups
            g = hb[off: off + nb].view(np.int32).copy()
            off += nb
            results.append(merge(q, g, hr) if split else g)
        return WindowRun(results, (done_at - st["t0"]) * 1e3, len(st["queries"]), len(st["segs"]),
                         len(st["gsegs"]), len(st["csegs"]), st["staged"], st["launches"], st["span"],
                         plan_ms=st["plan_ms"], gpu_ms=st["g0"].elapsed_time(st["g1"]), cpu_ms=st["cpu_ms"][0],
                         copied_column_segments=st["copied"], extra={"waves": st["waves"], "done_at": done_at})

    def run_window(self, queries: list[B.Query], planner) -> WindowRun:
        """One window on its own: planned, run and merged before returning."""
        return self._finish_window(self._start_window(queries, planner))

    def run(self, queries: list[B.Query], planner, window: int = 256) -> list[WindowRun]:
        """All queries in windows of `window`, in order. Window k + 1 is planned and
        enqueued while window k's copies, scans and CPU share run (its scans queue behind
        window k's on the kernel stream, its CPU share behind window k's on the CPU worker),
        so the host-to-device link and the host cores do not idle between windows."""
        runs, pending = [], None
        for i in range(0, len(queries), window):
            st = self._start_window(queries[i: i + window], planner)
            if pending is not None:
                runs.append(self._finish_window(pending))
            pending = st
        if pending is not None:
            runs.append(self._finish_window(pending))
        return runs
