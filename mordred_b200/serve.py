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
"""
from __future__ import annotations

import collections
import math
import statistics
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

    def summary(self, rows: int) -> dict:
        lat = sorted(self.latencies_ms)
        pct = lambda p: lat[min(len(lat) - 1, max(0, int(math.ceil(p * len(lat))) - 1))] if lat else None
        return {"queries": self.queries, "completed": len(lat), "seconds": self.seconds,
                "qps": len(lat) / self.seconds if self.seconds else None,
                "p50_ms": pct(0.50), "p90_ms": pct(0.90), "p99_ms": pct(0.99), "max_ms": lat[-1] if lat else None,
                "batches": self.batches, "mean_batch": statistics.mean(self.batch_sizes) if self.batch_sizes else 0,
                "mean_batch_ms": statistics.mean(self.batch_ms) if self.batch_ms else 0,
                "fact_rows_per_s": self.batches * rows / self.seconds if self.seconds else None,
                "query_rows_per_s": len(lat) * rows / self.seconds if self.seconds else None,
                "rejected": self.rejected, "deferred_admissions": self.deferred,
                "peak_admitted_bytes": self.peak_held_bytes}


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
              keep_results: bool = False) -> tuple[ServeReport, dict]:
        """Serve `queries` arriving at `arrivals` (s, ascending) in real time."""
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
                ac.arrive(i, nbytes[i])
                i += 1
            rep.peak_held_bytes = max(rep.peak_held_bytes, ac.held)
            batch = ac.take(self.max_batch)
            if not batch:
                if i < len(queries):
                    time.sleep(max(0.0, min(arrivals[i] - now, 0.001)))
                    continue
                if now > max_wait_s:
                    break
                continue
            b0 = time.perf_counter()
            res = self.run_batch([queries[qid] for qid, _ in batch])
            end = time.perf_counter() - t0
            rep.batches += 1
            rep.batch_sizes.append(len(batch))
            rep.batch_ms.append((time.perf_counter() - b0) * 1e3)
            for (qid, nb), r in zip(batch, res):
                rep.latencies_ms.append((end - arrivals[qid]) * 1e3)
                if keep_results:
                    results[qid] = r
                ac.release(nb)
            done += len(batch)
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
    args = ap.parse_args()
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    sizes = ssb.Sizes(lo_len=args.rows)
    t = ssb.gen_device(sizes, args.seed, B.BATCH_FACT, B.BATCH_DIMS)
    srv = Server(t, sizes, args.rows, int(args.budget_gb * (1 << 30)))
    n = int(args.rate * args.seconds)
    qs = B.generate_queries(n, seed=args.seed + 3)
    srv.run_batch(qs[:8])  # load the kernels
    rep, _ = srv.serve(qs, poisson_arrivals(args.rate, n, args.seed + 5))
    print(json.dumps(dict(rep.summary(args.rows), rows=args.rows, rate_qps=args.rate,
                          budget_bytes=srv.budget, device_status=L.device_status(0))), flush=True)


if __name__ == "__main__":
    main()
