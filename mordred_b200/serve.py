"""Serving loop: queries arrive as a Poisson stream; an admission controller caps the
device bytes that admitted queries hold; the server answers whatever is admitted and
waiting with one batched scan of the GPU-resident fact table (mb_batch_run, up to 256
queries a launch), over and over.

The reference has no serving loop (it runs queries from an interactive menu,
src/gpudb/main.cu:72-489, one at a time). Here:

* :class:`AdmissionController` — a query holds its result array and its share of the
  batch's query-mask workspace while queued or running; it is admitted only while the
  admitted total stays within the byte budget (and the queue within its length limit),
  else it waits in arrival order (never reordered, never dropped unless the wait limit
  passes).
* :class:`Server` — real-time loop on the host clock: arrivals are released at their
  Poisson times; whenever the GPU is idle the server takes every admitted waiting query
  (up to the batch limit), plans the batch, runs it and reads the results back. A
  query's latency is its batch's completion time minus its arrival time.
* :class:`CircularServer` — the table is cut into chunks that batched launches visit in
  a cycle; admitted queries join at the next launch and finish after one lap, so a
  query waits about one scan instead of the batch in progress plus its own.
* :class:`PlannerRouter` — the learned planner (or the analytic model) on the serving
  path: over a date-sorted table, an arriving query whose candidate segments the host
  cores can answer sooner than the GPU's queue would (predicted CPU ms plus the CPU
  queue's backlog, against the GPU latency the server is currently seeing) is answered
  by the CPU engine from the pinned host columns instead of joining a GPU batch, which
  also takes its work off the saturated GPU.
"""
from __future__ import annotations

import collections
import ctypes as C
import gc
import math
import queue
import statistics
import sys
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from . import batch as B
from . import ssb


def poisson_arrivals(rate_qps: float, n: int, seed: int) -> np.ndarray:
    """Arrival times (s) of n queries of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_qps, n))


def query_bytes(q: B.Query) -> int:
    """Device bytes a query holds: its result array plus its share of the per-batch mask
    tables (one 32-byte mask per value of each constrained attribute: at most 2,557
    date intervals and the small domains), rounded up to 4 KB."""
    res = 8 if q.template == "agg" else 16 * q.groups
    masks = (2 * 2557 + 11 + 50 + 5 * 3 + 25) * 32 // 256  # a 256-query batch's tables, per query
    return (res + masks + 4095) // 4096 * 4096


class AdmissionController:
    """FIFO admission under a byte budget and a queue-length limit."""

    def __init__(self, budget_bytes: int, max_queue: int = 100_000):
        self.budget = budget_bytes
        self.max_queue = max_queue
        self.held = 0
        self.waiting: collections.deque = collections.deque()   # (id, bytes) not yet admitted
        self.admitted: collections.deque = collections.deque()  # ids admitted, not yet running
        self.deferred = 0
        self.rejected = 0

    def arrive(self, qid: int, nbytes: int) -> bool:
        if len(self.waiting) + len(self.admitted) >= self.max_queue or nbytes > self.budget:
            self.rejected += 1
            return False
        self.waiting.append((qid, nbytes))
        self._admit()
        return True

    def _admit(self) -> None:
        while self.waiting and self.held + self.waiting[0][1] <= self.budget:
            qid, nb = self.waiting.popleft()
            self.held += nb
            self.admitted.append((qid, nb))
        if self.waiting:
            self.deferred += 1

    def take(self, limit: int) -> list[tuple[int, int]]:
        out = []
        while self.admitted and len(out) < limit:
            out.append(self.admitted.popleft())
        return out

    def release(self, nbytes: int) -> None:
        self.held -= nbytes
        self._admit()


@dataclass
class ServeReport:
    queries: int
    seconds: float
    latencies_ms: list = field(default_factory=list)
    batches: int = 0
    batch_sizes: list = field(default_factory=list)
    batch_ms: list = field(default_factory=list)
    rejected: int = 0
    deferred: int = 0
    peak_held_bytes: int = 0
    scan_rows: int = 0          # fact rows the launches scanned
    cpu_answered: int = 0       # queries the router sent to the host cores
    cap_raises: int = 0         # circular scan: times the active-set cap rose under a backlog

    def summary(self, rows: int) -> dict:
        lat = sorted(self.latencies_ms)
        pct = lambda p: lat[min(len(lat) - 1, max(0, int(math.ceil(p * len(lat))) - 1))] if lat else None
        return {"queries": self.queries, "completed": len(lat), "seconds": self.seconds,
                "qps": len(lat) / self.seconds if self.seconds else None,
                "p50_ms": pct(0.50), "p90_ms": pct(0.90), "p99_ms": pct(0.99), "max_ms": lat[-1] if lat else None,
                "batches": self.batches, "mean_batch": statistics.mean(self.batch_sizes) if self.batch_sizes else 0,
                "mean_batch_ms": statistics.mean(self.batch_ms) if self.batch_ms else 0,
                "fact_rows_per_s": (self.scan_rows or self.batches * rows) / self.seconds if self.seconds else None,
                "query_rows_per_s": len(lat) * rows / self.seconds if self.seconds else None,
                "rejected": self.rejected, "deferred_admissions": self.deferred,
                "peak_admitted_bytes": self.peak_held_bytes, "cpu_answered": self.cpu_answered,
                "cap_raises": self.cap_raises}


def _drain_cpu(router, rep: ServeReport, results: dict, queries, arrivals, t0: float, keep: bool) -> int:
    """Record the queries the router's CPU worker has finished; returns how many."""
    n = 0
    while router is not None:
        try:
            qid, res, tdone = router.done.get_nowait()
        except queue.Empty:
            break
        rep.latencies_ms.append((tdone - t0 - arrivals[qid]) * 1e3)
        rep.cpu_answered += 1
        if keep:
            results[qid] = res.view(np.int64).copy() if queries[qid].template == "agg" else res
        n += 1
    return n


class _paused_gc:
    """The cyclic garbage collector paused for a serving run (restored after). Everything
    the loop allocates per query and per launch is freed by reference counting, while a
    full collection walks every object of the process (host tables, thousands of queries)
    on the serving thread; one run of 4 s at 2,000 q/s showed a 0.5 s stall of that kind
    (p99 470 ms against 48-56 ms in the runs before and after it)."""

    def __enter__(self):
        self.was = gc.isenabled()
        gc.disable()

    def __exit__(self, *exc):
        if self.was:
            gc.enable()


def _arrive(ac, router, qid: int, q, nbytes: int) -> None:
    if router is None or not router.route(qid, q):
        ac.arrive(qid, nbytes)


class _AllResident:
    """The residency view of a table whose columns all live on the GPU."""

    def __init__(self, nseg: int, ncol: int):
        self.num_slots = nseg * ncol
        self._idx = np.zeros(nseg, np.int32)

    def col_idx(self, col: int) -> np.ndarray:
        return self._idx

    def stats(self) -> dict:
        return {"resident": self.num_slots}


class PlannerRouter:
    """Sheds load from a congested GPU: while the median latency of recent GPU completions
    exceeds `gpu_target_ms`, an arriving query over at most `max_segments` candidate
    segments goes to the host cores when the planner predicts they answer it sooner than
    the GPU path: predicted CPU ms over its candidate segments (segment
    skipping on the date-sorted table) plus the CPU queue's predicted backlog, against
    `margin` x the GPU latency the server has been seeing (a running median of recent GPU
    completions). The CPU side is one worker thread running queries one at a time on the
    CPU engine (mb_cpu_star_query over the pinned host columns, on `cpu_share` of the host
    threads); its results equal the GPU's (integer sums; rows outside the candidate
    segments cannot match the query's date range)."""

    def __init__(self, table, planner, margin: float = 0.5, max_backlog_ms: float = 50.0, cpu_share: float = 0.5,
                 max_segments: int = 24, gpu_target_ms: float = 100.0, max_inflight: int = 1):
        from .engine import FACT, CpuShare, host_tables

        class _Share(CpuShare):
            pass

        self.share = _Share()
        self.share.t = table
        self.share.hht = host_tables(table.sizes)
        self.share.cache = _AllResident(table.nseg, len(FACT))
        from . import cpu as _cpu
        # the serving thread (planning, launches, result copies) keeps the other threads: a
        # CPU engine on every core slows the GPU path it is meant to relieve (measured: GPU
        # batches took longer and latency rose with all host threads routed)
        self.share.cpu_nthreads = max(1, int(_cpu.threads() * cpu_share))
        self.share.cpu_threads = self.share.cpu_nthreads
        self.planner = planner
        # predictions on the host: a forward launch would queue behind the batch kernels
        self._predict = getattr(planner, "predict_host", planner.predict)
        self.margin = margin
        self.max_backlog_ms = max_backlog_ms
        # the decision runs on the serving thread for every arrival: queries over more
        # candidate segments than this are left to the GPU without consulting the model
        self.max_segments = max_segments
        # queries stay on the GPU while its median latency meets this target: below it,
        # the CPU engine's work on the host cores costs the GPU path more than the routed
        # queries gain (measured at 2,000 q/s: circular-scan p99 72-80 ms with every
        # eligible query routed, 52 ms with none)
        self.gpu_target_ms = gpu_target_ms
        # queries on the host cores at once: each one's engine threads and interpreter time
        # slow the serving thread, and under overload an unbounded queue fed itself (measured
        # at 2,800 q/s: p99 433 ms with routing against 64 ms without, one run in two); with
        # one at a time the CPU relieves the scan by at most its own rate
        self.max_inflight = max_inflight
        self.inflight = 0
        self.gpu_lat = collections.deque(maxlen=64)
        self.backlog_ms = 0.0
        self.q: queue.Queue = queue.Queue()
        self.done: queue.Queue = queue.Queue()
        self.routed = 0
        self.considered = 0
        self.pred_ms: list[float] = []
        self.cpu_ms: list[float] = []
        self._lock = threading.Lock()
        # the serving thread has to get the interpreter back within a fraction of one launch
        # (a few ms) whenever the worker runs Python between its engine calls; the default
        # 5 ms switch interval can hand the worker a whole launch's worth of time
        self._switch = sys.getswitchinterval()
        sys.setswitchinterval(min(self._switch, 2e-4))
        self._th = threading.Thread(target=self._worker, daemon=True)
        self._th.start()

    def note_gpu_latency(self, ms: float) -> None:
        self.gpu_lat.append(ms)

    def route(self, qid: int, q: B.Query) -> bool:
        """True when q was queued for the CPU (its result arrives through `done`)."""
        self.considered += 1
        if len(self.gpu_lat) < 8:
            return False  # no GPU latency seen yet
        gpu_now = float(np.median(self.gpu_lat))
        if gpu_now < self.gpu_target_ms:
            return False  # the GPU meets its latency target: no shedding
        if self.inflight >= self.max_inflight:
            return False  # the host cores are busy with earlier routed queries
        cand = self.share.candidates(q)
        if len(cand) > self.max_segments:
            return False
        if len(cand) == 0:
            pred = 0.0
        else:
            pc, pg, fc, fg = self._predict(self.share.context(q, cand))
            pred = float(np.sum(pc) + fc)
        with self._lock:
            if self.inflight >= self.max_inflight or self.backlog_ms + pred > min(self.margin * gpu_now,
                                                                                   self.max_backlog_ms):
                return False
            self.backlog_ms += pred
            self.inflight += 1
        self.routed += 1
        self.q.put((qid, q, cand, pred))
        return True

    def _worker(self) -> None:
        while True:
            item = self.q.get()
            if item is None:
                return
            qid, q, cand, pred = item
            c0 = time.perf_counter()
            res = np.zeros(2 if q.template == "agg" else 4 * q.groups, np.int32)
            if len(cand):
                self.share.build_cpu(q)
                self.share._cpu_segments(q, [int(x) for x in cand], res)
            ms = (time.perf_counter() - c0) * 1e3
            with self._lock:
                self.backlog_ms = max(0.0, self.backlog_ms - pred)
                self.inflight -= 1
                self.pred_ms.append(pred)
                self.cpu_ms.append(ms)
            self.done.put((qid, res, time.perf_counter()))

    def close(self) -> None:
        self.q.put(None)
        self._th.join(timeout=60)
        sys.setswitchinterval(self._switch)

    def summary(self) -> dict:
        err = [abs(math.log(max(p, 1e-3)) - math.log(max(m, 1e-3))) for p, m in zip(self.pred_ms, self.cpu_ms)]
        return {"planner": getattr(self.planner, "name", "?"), "routed_to_cpu": self.routed,
                "considered": self.considered,
                "cpu_ms_mean": statistics.mean(self.cpu_ms) if self.cpu_ms else None,
                "mae_log_ms_cpu_prediction": statistics.mean(err) if err else None}


class Server:
    """Answers queries over GPU-resident fact columns `t` (BATCH_FACT + dims) of n rows."""

    def __init__(self, t: dict, sizes: ssb.Sizes, n_rows: int, budget_bytes: int = 16 << 30,
                 max_batch: int = L.MB_BATCH_MAX_QUERIES):
        self.t, self.sizes, self.n = t, sizes, n_rows
        self.pats = B.build_pats(t, sizes)
        self.budget = budget_bytes
        self.max_batch = max_batch

    def run_batch(self, qs: list[B.Query]) -> list[np.ndarray]:
        flat, views = B.result_buffers(qs)
        B.BatchPlan(self.t, self.pats, qs, views, self.n).run()
        host = flat.cpu()  # waits for the batch
        out, off = [], 0
        for q in qs:
            nb = 8 if q.template == "agg" else 16 * q.groups
            out.append(host[off: off + nb].numpy().view(np.int64 if q.template == "agg" else np.int32).copy())
            off += nb
        return out

    def serve(self, queries: list[B.Query], arrivals: np.ndarray, max_wait_s: float = 60.0,
              keep_results: bool = False, router: "PlannerRouter | None" = None) -> tuple[ServeReport, dict]:
        """Serve `queries` arriving at `arrivals` (s, ascending) in real time (see _serve),
        with the cyclic garbage collector paused for the run."""
        with _paused_gc():
            return self._serve(queries, arrivals, max_wait_s, keep_results, router)

    def _serve(self, queries: list[B.Query], arrivals: np.ndarray, max_wait_s: float = 60.0,
               keep_results: bool = False, router: "PlannerRouter | None" = None) -> tuple[ServeReport, dict]:
        """Serve `queries` arriving at `arrivals` (s, ascending) in real time; with a router,
        queries it sends to the host cores bypass the GPU batches."""
        ac = AdmissionController(self.budget)
        rep = ServeReport(len(queries), 0.0)
        results = {}
        nbytes = [query_bytes(q) for q in queries]
        done = 0
        i = 0
        t0 = time.perf_counter()
        while done + ac.rejected < len(queries):
            now = time.perf_counter() - t0
            while i < len(queries) and arrivals[i] <= now:
                _arrive(ac, router, i, queries[i], nbytes[i])
                i += 1
            done += _drain_cpu(router, rep, results, queries, arrivals, t0, keep_results)
            rep.peak_held_bytes = max(rep.peak_held_bytes, ac.held)
            batch = ac.take(self.max_batch)
            if not batch:
                if i < len(queries):
                    time.sleep(max(0.0, min(arrivals[i] - now, 0.001)))
                    continue
                if now > max_wait_s:
                    break
                time.sleep(0.0002)  # only CPU-routed queries are outstanding
                continue
            b0 = time.perf_counter()
            res = self.run_batch([queries[qid] for qid, _ in batch])
            end = time.perf_counter() - t0
            rep.batches += 1
            rep.batch_sizes.append(len(batch))
            rep.batch_ms.append((time.perf_counter() - b0) * 1e3)
            for (qid, nb), r in zip(batch, res):
                rep.latencies_ms.append((end - arrivals[qid]) * 1e3)
                if router is not None:
                    router.note_gpu_latency((end - arrivals[qid]) * 1e3)
                if keep_results:
                    results[qid] = r
                ac.release(nb)
            done += len(batch)
        rep.seconds = time.perf_counter() - t0
        rep.rejected, rep.deferred = ac.rejected, ac.deferred
        return rep, results


@dataclass
class _Member:
    qid: int
    nbytes: int
    query: B.Query
    cq: L.MbBatchQuery          # the query's launch descriptor, made once at admission
    res: torch.Tensor           # its device result, accumulated over the chunks
    pending: np.ndarray = None  # per chunk: still to be launched for it (bool)
    left: int = 0               # chunks still to be launched for it


class CircularServer:
    """Cooperative circular scan: the GPU-resident table is split into `chunks` row
    ranges that one batched launch after another visits in a cycle. An admitted query
    joins the running scan at the next launch and completes once every chunk it needs has
    been launched for it (within one lap from wherever it joined), so it waits for about
    one scan of the table rather than for the batch in progress plus its own. Every query
    sees every row it needs exactly once and the kernel only adds into its result, so
    results are those of the query run alone. Up to 256 queries share a launch; a second
    launch is queued before the first completes so the GPU never waits for the host.

    Chunk skipping (`skip`, the planner's segment skipping, QueryOptimizer.cu:1641-1662):
    each chunk's orderdate [min, max] is taken when the server starts; a query needs only
    the chunks whose range meets its date range (rows elsewhere cannot pass its date
    predicate), and the scan moves on to the next chunk some active query needs, so on a
    date-sorted table a query over a few weeks costs one chunk's launch, not a lap, and
    chunks no active query needs are not scanned at all."""

    # Load-following cap on the active set. Up to 128 queries a launch carry 4 words of query
    # mask per attribute value and more carry 8, which doubles every row's mask work; below
    # saturation the scan therefore keeps at most `max_active` (128) queries, so that a burst
    # cannot tip it into the slower 8-word launches. When admitted queries have waited longer
    # than one lap for a place (the 128-query scan answers fewer queries per second than
    # arrive), the cap rises to `burst_active` (256): a lap then costs more but answers twice
    # the queries, so the backlog drains instead of growing without bound. The cap falls
    # back once nothing waits and the active set is back within `max_active`.
    def __init__(self, t: dict, sizes: ssb.Sizes, n_rows: int, budget_bytes: int = 16 << 30,
                 max_active: int = 128, chunks: int = 8, burst_active: int = L.MB_BATCH_MAX_QUERIES,
                 skip: bool = True):
        self.t, self.sizes, self.n = t, sizes, n_rows
        self.pats = B.build_pats(t, sizes)
        self.dims = self.pats.c_dims()
        self.budget = budget_bytes
        self.max_active = max_active
        self.burst_active = max(max_active, burst_active)
        step = -(-n_rows // max(1, chunks))
        step = -(-step // 4096) * 4096  # 16-byte aligned chunk starts
        self.bounds = [(r0, min(n_rows, r0 + step)) for r0 in range(0, n_rows, step)] or [(0, 0)]
        self.ws = torch.empty(16, dtype=torch.uint8, device=next(iter(t.values())).device)
        self.skip = skip
        od = t["lo_orderdate"]
        rng = [torch.aminmax(od[r0:r1]) if r1 > r0 else (torch.tensor(1), torch.tensor(0)) for r0, r1 in self.bounds]
        self.chunk_lo = np.array([int(lo) for lo, _ in rng], np.int64)
        self.chunk_hi = np.array([int(hi) for _, hi in rng], np.int64)

    def chunks_needed(self, q: B.Query) -> np.ndarray:
        """Per chunk, whether q can have a matching row in it (all chunks without skipping)."""
        if not self.skip:
            return np.ones(len(self.bounds), bool)
        return (self.chunk_hi >= q.date[0]) & (self.chunk_lo <= q.date[1])

    def _launch(self, c: int, members: list) -> None:
        r0, r1 = self.bounds[c]
        arr = (L.MbBatchQuery * len(members))(*[m.cq for m in members])
        a = L.MbBatchArgs()
        a.num_rows = r1 - r0
        for i, name in enumerate(B.BATCH_FACT):
            col = self.t[name]
            a.fact[i] = col.data_ptr() + r0 * col.element_size()
        a.dim = self.dims
        a.num_queries = len(members)
        a.queries = C.cast(arr, C.POINTER(L.MbBatchQuery))
        a.smem_group_bytes = -1
        need = int(L.lib().mb_batch_workspace_bytes(C.byref(a)))
        if need > self.ws.numel():
            torch.cuda.current_stream().synchronize()  # launches in flight use the old workspace
            self.ws = torch.empty(max(need, 2 * self.ws.numel()), dtype=torch.uint8, device=self.ws.device)
        a.workspace, a.workspace_bytes = self.ws.data_ptr(), self.ws.numel()
        L.check("mb_batch_run", L.lib().mb_batch_run(C.byref(a), ssb._stream()))

    def serve(self, queries: list[B.Query], arrivals: np.ndarray, max_wait_s: float = 60.0,
              keep_results: bool = False, router: "PlannerRouter | None" = None) -> tuple[ServeReport, dict]:
        """Serve `queries` arriving at `arrivals` (s, ascending) in real time (see _serve),
        with the cyclic garbage collector paused for the run."""
        with _paused_gc():
            return self._serve(queries, arrivals, max_wait_s, keep_results, router)

    def _serve(self, queries: list[B.Query], arrivals: np.ndarray, max_wait_s: float = 60.0,
               keep_results: bool = False, router: "PlannerRouter | None" = None) -> tuple[ServeReport, dict]:
        """Serve `queries` arriving at `arrivals` (s, ascending) in real time; with a router,
        queries it sends to the host cores bypass the scan."""
        ac = AdmissionController(self.budget)
        rep = ServeReport(len(queries), 0.0)
        results = {}
        nbytes = [query_bytes(q) for q in queries]
        nchunks = len(self.bounds)
        active: list[_Member] = []            # still have chunks to be launched
        instant: list[_Member] = []           # need no chunk: complete at admission
        inflight: collections.deque = collections.deque()  # (event, members finishing with it, launch time)
        c = 0
        done = 0
        i = 0
        cap = self.max_active
        lap_s = None               # duration of the last lap of the scan position (s)
        lap_start, last_c = None, -1
        t0 = time.perf_counter()
        while done + ac.rejected < len(queries):
            now = time.perf_counter() - t0
            while i < len(queries) and arrivals[i] <= now:
                _arrive(ac, router, i, queries[i], nbytes[i])
                i += 1
            done += _drain_cpu(router, rep, results, queries, arrivals, t0, keep_results)
            # the cap follows the load: raised while the oldest admitted query has waited
            # for a place longer than a lap, lowered when the backlog is gone
            if ac.admitted and lap_s is not None and cap < self.burst_active:
                if now - arrivals[ac.admitted[0][0]] > lap_s:
                    cap = self.burst_active
                    rep.cap_raises += 1
            elif not ac.admitted and cap > self.max_active and len(active) <= self.max_active:
                cap = self.max_active
            for qid, nb in ac.take(cap - len(active)):
                res = queries[qid].result_buffer()
                need = self.chunks_needed(queries[qid])
                m = _Member(qid, nb, queries[qid], queries[qid].to_c(res), res, need.copy(), int(need.sum()))
                (active if m.left else instant).append(m)
            if instant:
                # no chunk can hold a matching row: the (zeroed) result is the answer
                end = time.perf_counter() - t0
                for m in instant:
                    if keep_results:
                        results[m.qid] = m.res.cpu().numpy().reshape(-1).view(
                            np.int64 if m.query.template == "agg" else np.int32).copy()
                    rep.latencies_ms.append((end - arrivals[m.qid]) * 1e3)
                    ac.release(m.nbytes)
                done += len(instant)
                instant = []
            rep.peak_held_bytes = max(rep.peak_held_bytes, ac.held)
            if active and len(inflight) < 2:
                # the next chunk (cyclically from the scan position) some active query needs
                want = np.zeros(nchunks, bool)
                for m in active:
                    want |= m.pending
                step = int(np.argmax(np.roll(want, -c)))
                c = (c + step) % nchunks
                if lap_start is None or c <= last_c:  # the scan position wrapped: a lap ends
                    tl = time.perf_counter()
                    if lap_start is not None:
                        lap_s = tl - lap_start
                    lap_start = tl
                last_c = c
                members = [m for m in active if m.pending[c]]
                self._launch(c, members)
                ev = torch.cuda.Event()
                ev.record()
                finishing = []
                for m in members:
                    m.pending[c] = False
                    m.left -= 1
                    if m.left == 0:
                        finishing.append(m)
                active = [m for m in active if m.left > 0]
                inflight.append((ev, finishing, time.perf_counter()))
                rep.batches += 1
                rep.batch_sizes.append(len(members))
                rep.scan_rows += self.bounds[c][1] - self.bounds[c][0]
                c = (c + 1) % nchunks
                continue
            if inflight:
                ev, finishing, tl = inflight.popleft()
                ev.synchronize()
                end = time.perf_counter() - t0
                rep.batch_ms.append((time.perf_counter() - tl) * 1e3)
                if finishing:
                    host = torch.cat([m.res.reshape(-1).view(torch.uint8) for m in finishing]).cpu()
                    off = 0
                    for m in finishing:
                        nb = m.res.numel() * m.res.element_size()
                        if keep_results:
                            results[m.qid] = host[off: off + nb].numpy().view(
                                np.int64 if m.query.template == "agg" else np.int32).copy()
                        off += nb
                        rep.latencies_ms.append((end - arrivals[m.qid]) * 1e3)
                        if router is not None:
                            router.note_gpu_latency((end - arrivals[m.qid]) * 1e3)
                        ac.release(m.nbytes)
                    done += len(finishing)
                continue
            if i < len(queries):
                time.sleep(max(0.0, min(arrivals[i] - now, 0.001)))
            elif now > max_wait_s:
                break
            else:
                time.sleep(0.0002)  # only CPU-routed queries are outstanding
        rep.seconds = time.perf_counter() - t0
        rep.rejected, rep.deferred = ac.rejected, ac.deferred
        return rep, results


def main():
    import argparse
    import json

    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=600_000_000)
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--seconds", type=float, default=5.0)
    ap.add_argument("--seed", type=int, default=20260101)
    ap.add_argument("--budget-gb", type=float, default=16.0)
    ap.add_argument("--chunks", type=int, default=0, help="circular scan over this many chunks (0: whole-scan batches)")
    args = ap.parse_args()
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    sizes = ssb.Sizes(lo_len=args.rows)
    t = ssb.gen_device(sizes, args.seed, B.BATCH_FACT, B.BATCH_DIMS)
    budget = int(args.budget_gb * (1 << 30))
    srv = CircularServer(t, sizes, args.rows, budget, chunks=args.chunks) if args.chunks else \
        Server(t, sizes, args.rows, budget)
    n = int(args.rate * args.seconds)
    qs = B.generate_queries(n, seed=args.seed + 3)
    (srv if isinstance(srv, Server) else Server(t, sizes, args.rows, budget)).run_batch(qs[:8])  # load kernels
    rep, _ = srv.serve(qs, poisson_arrivals(args.rate, n, args.seed + 5))
    print(json.dumps(dict(rep.summary(args.rows), rows=args.rows, rate_qps=args.rate, chunks=args.chunks,
                          budget_bytes=srv.budget, device_status=L.device_status(0))), flush=True)


if __name__ == "__main__":
    main()
