"""Benchmark: star join + group-by (Query A and Query B) over a 120,000,000-row fact table.

One step = Query A (3 filtered PHT builds + the fused supplier->part->date probe with
the 7x1000 group-by) and Query B (4 builds + the fused 4-way probe with the 7x25
group-by), each over every fact row. value = fact rows processed per second
(2 x 120 M per step per GPU). Inputs are synthetic (seeded generator with the
configured shapes) and larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Beside the headline the line reports, outside the timed steps: the filter-aggregate
(16 B/row) on the full table and on its own 6 M-row table with L2 flushed; and a batch
of 256 generated queries run as one shared scan (CUDA graph replay) against the same
queries run one at a time, with the results compared bit for bit; and (at N = 1) the
learned planner against the analytic cost model over a 600 M-row host-resident table
with an 8 GB GPU segment cache: end-to-end ms of the same queries and the prediction
error of each model; and (at N = 1) the serving loop: Poisson arrivals at 2,000 q/s over
a 600 M-row GPU-resident table, p50/p99 latency, q/s and fact rows/s.

N > 1 runs under torchrun: rank r holds rows [r*120M, (r+1)*120M) of one table
(weak scaling), and each step all-reduces the dense group sums over NCCL.
The reference arm (--impl reference) times the reference's own CPU engine
(src/cpu/ssb/q21.cpp and q41.cpp built under oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fact rows/s (GB/s vs HBM peak) per star query; learned vs plain planner ms"
UNIT = "fact rows/s"
LO_LEN = 120_000_000
SEED = 20260101
QA_BYTES_PER_ROW = 16   # suppkey, partkey, orderdate, revenue
QB_BYTES_PER_ROW = 24   # + custkey, supplycost


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=LO_LEN)
    ap.add_argument("--cpu-sample-rows", type=int, default=24_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-planner", action="store_true")
    ap.add_argument("--planner-rows", type=int, default=600_000_000)
    ap.add_argument("--planner-queries", type=int, default=2000)
    ap.add_argument("--batch-queries", type=int, default=256)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-rows", type=int, default=600_000_000)
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-seconds", type=float, default=4.0)
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle reasons of one GPU, polled through NVML every 5 ms while the
    timed region runs (short enough to sample a region of a few tens of milliseconds)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4}

    def __init__(self, device: int):
        self.device = device
        self.samples: list[tuple[int, int]] = []
        self.max_mhz = None
        self.error = None
        self._stop = threading.Event()
        self._t = None

    def _handle(self):
        import pynvml as N
        import torch

        N.nvmlInit()
        try:
            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return N.nvmlDeviceGetHandleByIndex(self.device)

    def _run(self, h):
        import pynvml as N

        while not self._stop.is_set():
            try:
                self.samples.append((N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM),
                                     N.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception as e:  # keep what was sampled
                self.error = str(e)
                return
            self._stop.wait(0.005)

    def __enter__(self):
        try:
            import pynvml as N

            h = self._handle()
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            self._t = threading.Thread(target=self._run, args=(h,), daemon=True)
            self._t.start()
        except Exception as e:
            self.error = str(e)
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=2)

    def summary(self):
        sm = [c for c, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS.items() if r & bit})
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
               "samples": len(sm), "source": "NVML, 5 ms polling during the timed region"}
        if self.error:
            out["error"] = self.error
        return out


def cpu_baseline_reference(rows: int, trials: int, threads: int = 0):
    """Time the reference's own CPU engine (oracle/_ref) on `rows` fact rows; returns
    (rows/s, cores, per-trial step ms)."""
    from oracle import oracle as O

    cores = threads or os.cpu_count() or 1
    _, ms21 = O.run_ref(21, SEED, rows, 40_000, 600_000, 1_000_000, 2556, trials=trials, threads=cores,
                        timeout=1800)
    _, ms41 = O.run_ref(41, SEED, rows, 40_000, 600_000, 1_000_000, 2556, trials=trials, threads=cores,
                        timeout=1800)
    steps = [a + b for a, b in zip(ms21, ms41)]
    return steps, cores


def cpu_baseline_port(rows: int, trials: int):
    """Time the C oracle restatement (all host threads) on `rows` fact rows."""
    from mordred_b200 import ssb
    from oracle import oracle as O

    s = ssb.Sizes(lo_len=rows)
    h = ssb.gen_host(s, SEED, ssb.QB_FACT, sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    steps = []
    for _ in range(trials):
        t0 = time.perf_counter()
        O.q21(h, ssb.DATE_SLOTS)
        O.q41(h, ssb.DATE_SLOTS)
        steps.append((time.perf_counter() - t0) * 1e3)
    return steps, os.cpu_count() or 1


def filter_aggregate_full(t, n, ws, reps=20):
    """Median CUDA-event time of the filter-aggregate over the whole resident table."""
    import torch

    from mordred_b200 import ssb

    ms = []
    for _ in range(reps + 2):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ssb.q11(t, n, ws, zero=False)
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms[2:])


def filter_aggregate_6m(s, rank, peak, copies=20, rows=6_000_000, reps=10):
    """Config 1: the filter-aggregate on 6,000,000-row tables, each launch reading a table of
    its own (copies x 96 MB, larger than L2 together) in a CUDA graph of back-to-back
    launches; results checked against the first direct run of each copy."""
    import torch

    from mordred_b200 import _lib as L
    from mordred_b200 import ssb

    st = ssb._stream()
    tabs = []
    for k in range(copies):
        tk = {}
        for name in ssb.Q11_COLUMNS:
            buf = torch.empty(rows, dtype=torch.int32, device="cuda")
            L.call("mb_gen_fact_column", ssb.FACT_COLUMNS[name], SEED + 1000 + k, rank * rows, rows, s.s_len, s.c_len,
                   s.p_len, ssb._p(buf), st)
            tk[name] = buf
        tabs.append(tk)
    rev = torch.zeros(copies, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(copies, dtype=torch.int32, device="cuda")

    def launch_all():
        for k, tk in enumerate(tabs):
            L.call("mb_q11_query", ssb._p(tk["lo_orderdate"]), ssb._p(tk["lo_discount"]), ssb._p(tk["lo_quantity"]),
                   ssb._p(tk["lo_extendedprice"]), rows, rev[k:].data_ptr(), cnt[k:].data_ptr(), ssb._stream())

    launch_all()
    torch.cuda.synchronize()
    first = rev.clone()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rev.zero_()
        cnt.zero_()
        launch_all()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    equal = bool(torch.equal(rev, first))
    per_launch = e0.elapsed_time(e1) / (reps * copies)
    # the same launches one by one, each after a 512 MB write and a 512 MB read of other
    # buffers (cold L2): the latency of one query on its own, launch overhead included
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    clean = torch.ones(128 << 20, dtype=torch.int32, device="cuda")
    sink = torch.zeros(1, dtype=torch.int64, device="cuda")
    cold = []
    for k in range(min(copies, 12)):
        flush.zero_()
        sink.add_(clean.sum(dtype=torch.int64))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        L.call("mb_q11_query", ssb._p(tabs[k]["lo_orderdate"]), ssb._p(tabs[k]["lo_discount"]),
               ssb._p(tabs[k]["lo_quantity"]), ssb._p(tabs[k]["lo_extendedprice"]), rows, rev[k:].data_ptr(),
               cnt[k:].data_ptr(), ssb._stream())
        b.record()
        torch.cuda.synchronize()
        cold.append(a.elapsed_time(b))
    del g, flush, clean, tabs
    torch.cuda.empty_cache()
    gbs = rows * 16 / per_launch / 1e6
    cold_ms = statistics.median(cold[2:])
    return {"rows": rows, "ms": per_launch, "fact_rows_per_s": rows / (per_launch / 1e3), "gbs": gbs,
            "frac_of_hbm": gbs / peak, "results_equal_direct_run": equal,
            "l2": f"{copies} separate {rows:,}-row tables ({copies * rows * 16 / 1e9:.2f} GB) in turn, CUDA graph of "
                  f"{copies} back-to-back launches, {reps} replays",
            "cold_single_launch": {"ms": cold_ms, "frac_of_hbm": rows * 16 / cold_ms / 1e6 / peak,
                                   "l2": "512 MB write then 512 MB read of other buffers before each launch"}}


def batch_section(t, s, n, rank, world, args):
    """256 generated queries (filter-aggregate, Query A and Query B forms; selectivities
    log-uniform in [1e-5, 0.3]) over this rank's fact rows: one batched scan, replayed
    from a CUDA graph, against running the queries one at a time (filtered builds + the
    fused probe per query, the reference's way). Results are compared bit for bit."""
    import torch
    import torch.distributed as dist

    from mordred_b200 import _lib as L
    from mordred_b200 import batch as B
    from mordred_b200 import ssb

    st = ssb._stream()
    for name in B.BATCH_FACT:
        if name not in t:
            buf = torch.empty(n, dtype=torch.int32, device="cuda")
            L.call("mb_gen_fact_column", ssb.FACT_COLUMNS[name], SEED, rank * n, n, s.s_len, s.c_len, s.p_len,
                   ssb._p(buf), st)
            t[name] = buf
    t.update(ssb.gen_device(s, SEED, [], [d for d in B.BATCH_DIMS if d not in t]))
    pats = B.build_pats(t, s)
    qs = B.generate_queries(args.batch_queries, seed=SEED)
    flat, views = B.result_buffers(qs)
    plan = B.BatchPlan(t, pats, qs, views, n)
    graph = plan.capture(zero=flat)
    for _ in range(3):
        graph.replay()
    reps = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    batch_ms = e0.elapsed_time(e1) / reps
    ws = B.AloneWorkspace(s)
    alone = [q.result_buffer() for q in qs]

    def one_at_a_time():
        for r in alone:
            r.zero_()
        for q, r in zip(qs, alone):
            B.run_alone(t, ws, q, r, n)

    one_at_a_time()
    torch.cuda.synchronize()
    a_reps = 2
    e0.record()
    for _ in range(a_reps):
        one_at_a_time()
    e1.record()
    torch.cuda.synchronize()
    alone_ms = e0.elapsed_time(e1) / a_reps
    equal = all(torch.equal(a.view(-1), b.view(-1)) for a, b in zip(views, alone))
    tm = torch.tensor([batch_ms, alone_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    batch_ms, alone_ms = float(tm[0]), float(tm[1])
    del graph
    cols = len(B.BATCH_FACT)
    peak, peak_kind = measured_peaks()
    return {"queries": len(qs), "fact_rows_per_gpu": n, "templates": {k: sum(q.template == k for q in qs)
                                                                      for k in ("agg", "qa", "qb")},
            "expected_matches_per_row": sum(q.meta["expected_selectivity"] for q in qs),
            "batched_ms": batch_ms, "one_at_a_time_ms": alone_ms, "speedup": alone_ms / batch_ms,
            "query_rows_per_s": len(qs) * n * world / (batch_ms / 1e3),
            "shared_scan_gbs": cols * 4 * n / batch_ms / 1e6, "shared_scan_frac_of_hbm": cols * 4 * n / batch_ms / 1e6 / peak,
            "peak_kind": peak_kind, "results_equal_one_at_a_time": equal,
            "launch": "CUDA graph replay (result memset + mask kernel + batch kernel)", "seed": SEED}


def planner_section(args, table=None):
    """Config 3: a host-resident, date-sorted fact table of --planner-rows rows (1 Mi-row
    segments, per-segment min/max) under an 8 GB GPU segment-cache budget, and
    --planner-queries generated queries. The plain form runs them one at a time (the
    reference's executor) with the analytic cost model and with the learned model; the
    batched form runs them in windows of 256 through the batched executor (shared scans,
    planner-driven placement and admission, staged streaming) with each model. Every form
    starts from the same cache contents; results are compared bit for bit across forms.
    Plus the mean absolute error of each model's log-ms predictions on segments profiled
    live here, and on the training log's hold-out."""
    import numpy as np
    import torch

    from mordred_b200 import batch as B
    from mordred_b200 import planner_experiment as PE
    from mordred_b200.batch_engine import BatchExecutor
    from mordred_b200.engine import SEG, Executor, SegmentedTable
    from mordred_b200.planner import MIN_MS, AnalyticPlanner, LearnedPlanner

    if not os.path.exists(PE.DEFAULT_WEIGHTS):
        return {"unavailable": "no trained planner weights in mordred_b200/planner_weights"}
    learned = LearnedPlanner.load(PE.DEFAULT_WEIGHTS)
    t0 = time.perf_counter()
    if table is None:
        table = SegmentedTable(args.planner_rows, SEED)
    slots = int(8 * (1 << 30) // (SEG * 4))
    setup_s = time.perf_counter() - t0
    queries = B.generate_queries(args.planner_queries, seed=SEED + 7)
    start = PE.initial_weights(table, queries)
    plain_res, batch_res = {}, {}
    ex = Executor(table, cache_slots=slots)
    plain = PE.evaluate(ex, [AnalyticPlanner(), learned], queries, start, log=lambda *a: None,
                        keep_results=plain_res)
    # live prediction error on freshly profiled segments (a different query seed)
    rng = np.random.default_rng(SEED + 11)
    feats, truth, ana = [], [], []
    for q in B.generate_queries(40, seed=SEED + 13):
        cand = ex.candidates(q)
        if len(cand) == 0:
            continue
        recs, _ = ex.profile_segments(q, rng.choice(cand, min(16, len(cand)), replace=False))
        for r in recs:
            feats.append(r["features"])
            truth.append([r["cpu_ms"], r["gpu_ms"]])
            ana.append([r["analytic_cpu_ms"], r["analytic_gpu_ms"]])
    truth = np.log(np.maximum(np.array(truth), MIN_MS))
    live = {"samples": len(feats),
            "learned": PE.mae_report(learned.predict_log(np.stack(feats)), truth),
            "analytic": PE.mae_report(np.log(np.maximum(np.array(ana), MIN_MS)), truth)}
    ex.cache.close()
    del ex
    torch.cuda.empty_cache()
    bx = BatchExecutor(table, cache_slots=slots)
    batched = PE.evaluate_batched(bx, [AnalyticPlanner(), learned], queries, start, log=lambda *a: None,
                                  keep_results=batch_res)
    # the whole workload as one window: every staged segment is copied once for all the
    # queries (up to 256 a launch) instead of once per window of 256
    whole_res = {}
    one_window = PE.evaluate_batched(bx, [AnalyticPlanner(), learned], queries, start, window=len(queries),
                                     log=lambda *a: None, keep_results=whole_res)
    bx.close()
    bx.cache.close()
    del bx
    torch.cuda.empty_cache()
    ref = plain_res["analytic"]
    identical = all(all(np.array_equal(a, b) for a, b in zip(ref, r)) for r in
                    [plain_res["learned"], batch_res["analytic"], batch_res["learned"], whole_res["analytic"],
                     whole_res["learned"]])
    base = plain["analytic"]["total_ms"]
    return {"fact_rows": args.planner_rows, "segments": table.nseg, "cache_slots": slots,
            "queries": len(queries), "setup_s": setup_s,
            "plain_analytic_ms": base, "plain_learned_ms": plain["learned"]["total_ms"],
            "batched_analytic_ms": batched["analytic"]["total_ms"],
            "batched_learned_ms": batched["learned"]["total_ms"],
            "batched_analytic_one_window_ms": one_window["analytic"]["total_ms"],
            "batched_learned_one_window_ms": one_window["learned"]["total_ms"],
            "speedup_batched_learned_one_window_vs_plain_analytic": base / one_window["learned"]["total_ms"],
            "speedup_batched_learned_vs_plain_analytic": base / batched["learned"]["total_ms"],
            "speedup_learned_vs_analytic_plain": base / plain["learned"]["total_ms"],
            "speedup_learned_vs_analytic_batched": batched["analytic"]["total_ms"] / batched["learned"]["total_ms"],
            "one_at_a_time": {k: plain[k] for k in ("analytic", "learned")},
            "batched": batched, "batched_one_window": one_window, "results_identical_all_forms": identical,
            "prediction_mae_live": live, "prediction_mae_training_holdout": learned.manifest.get("holdout"),
            "weights": "mordred_b200/planner_weights/mlp.bin", "seed": SEED}


def serve_section(args, table=None):
    """Config 5, the serving loop: Poisson arrivals at --serve-rate over a GPU-resident,
    date-sorted table of --serve-rows rows, a 16 GB admission budget, the batched kernel.
    Two GPU servers — whole-scan batches (up to 256 queries a launch) and the circular scan
    (admitted queries join the running scan at the next of 8 chunks and complete after one
    lap; at most 128 at a time, 256 while a backlog waits longer than a lap) — each with
    the learned planner's router, which sheds queries the host cores answer sooner to the
    CPU engine once the GPU misses its latency target; over three arrival seeds, once
    without the router, and once at 1.4x the rate (circular scan, router on and off).
    Latency: arrival to completion. Results are checked against the queries run alone for
    a sample."""
    import numpy as np
    import torch

    from mordred_b200 import batch as B
    from mordred_b200 import planner_experiment as PE
    from mordred_b200 import serve as S
    from mordred_b200 import ssb
    from mordred_b200.engine import SegmentedTable
    from mordred_b200.planner import LearnedPlanner

    if table is None or table.n != args.serve_rows:
        table = SegmentedTable(args.serve_rows, SEED)
    sizes = table.sizes
    t = {k: torch.empty(table.n, dtype=torch.int32, device="cuda") for k in B.BATCH_FACT}
    for k in B.BATCH_FACT:
        t[k].copy_(table.host_t[k])
    t.update(table.dims)
    t.update(ssb.gen_device(sizes, SEED, [], [d for d in B.BATCH_DIMS if d not in t]))
    n = int(args.serve_rate * args.serve_seconds)
    planner = LearnedPlanner.load(PE.DEFAULT_WEIGHTS) if os.path.exists(PE.DEFAULT_WEIGHTS) else None
    whole = S.Server(t, sizes, table.n, 16 << 30)
    circ = S.CircularServer(t, sizes, table.n, 16 << 30, chunks=8)
    whole.run_batch(B.generate_queries(8, seed=1))
    # the circular scan's first launches allocate its workspace and page in its kernels: a
    # short run before the timed ones, so that a router never sees cold-start latencies
    circ.serve(B.generate_queries(64, seed=2), S.poisson_arrivals(args.serve_rate, 64, 5))
    keys = ("qps", "p50_ms", "p90_ms", "p99_ms", "max_ms", "batches", "mean_batch", "mean_batch_ms", "cpu_answered")
    runs = {"whole": [], "circular": []}
    routing = []
    checked = 0
    for k, seed in enumerate((SEED + 3, SEED + 31, SEED + 57)):
        qs = B.generate_queries(n, seed=seed)
        arrivals = S.poisson_arrivals(args.serve_rate, n, seed + 2)
        for name, srv in (("whole", whole), ("circular", circ)):
            router = S.PlannerRouter(table, planner) if planner is not None else None
            rep, _ = srv.serve(qs, arrivals, router=router)
            if router is not None:
                routing.append(router.summary())
                router.close()
            summ = rep.summary(table.n)
            runs[name].append({kk: summ[kk] for kk in keys})
            if k == 0:
                # results are checked on a separate, untimed run: keeping them copies each
                # answer to the host as it completes, which waits for the launches queued
                # behind it
                router = S.PlannerRouter(table, planner) if planner is not None else None
                _, res = srv.serve(qs, arrivals, router=router, keep_results=True)
                if router is not None:
                    router.close()
                ws = B.AloneWorkspace(sizes)
                for qid in range(0, n, max(1, n // 40)):
                    r = qs[qid].result_buffer()
                    B.run_alone(t, ws, qs[qid], r, table.n)
                    exp = r.cpu().numpy().reshape(-1)
                    got = np.asarray(res[qid]).reshape(-1)
                    assert np.array_equal(got.view(exp.dtype), exp), (name, qid)
                    checked += 1
    # the same first arrivals without the router: every query on the GPU
    qs = B.generate_queries(n, seed=SEED + 3)
    arrivals = S.poisson_arrivals(args.serve_rate, n, SEED + 5)
    no_router = {}
    for name, srv in (("whole", whole), ("circular", circ)):
        rep, _ = srv.serve(qs, arrivals)
        summ = rep.summary(table.n)
        no_router[name] = {kk: summ[kk] for kk in keys}
    # overload: 1.4x the rate on the circular scan, with the router shedding load to the
    # host cores and without it
    stress_rate = 1.4 * args.serve_rate
    n2 = int(stress_rate * args.serve_seconds)
    qs2 = B.generate_queries(n2, seed=SEED + 7)
    arr2 = S.poisson_arrivals(stress_rate, n2, SEED + 9)
    stress = {"rate_qps": stress_rate}
    for label, use in (("router", True), ("no_router", False)):
        router = S.PlannerRouter(table, planner) if use and planner is not None else None
        rep, _ = circ.serve(qs2, arr2, router=router)
        if router is not None:
            router.close()
        summ = rep.summary(table.n)
        stress[label] = {kk: summ[kk] for kk in keys + ("cap_raises",)}
    skipping = circ.skip
    del whole, circ, t
    torch.cuda.empty_cache()
    p99 = lambda name: [r["p99_ms"] for r in runs[name]]
    return {"rows": table.n, "rate_qps": args.serve_rate, "seconds_per_run": args.serve_seconds,
            "budget_bytes": 16 << 30, "table": "date-sorted, GPU-resident (9 fact columns)",
            "circular_chunk_skipping": skipping,
            "selectivity": "log-uniform in [1e-5, 0.3]", "seeds": 3, "router": "learned planner" if planner else None,
            "whole_scan_batches": runs["whole"], "circular_scan_8_chunks_max_128_active": runs["circular"],
            "p99_ms_whole_by_seed": p99("whole"), "p99_ms_circular_by_seed": p99("circular"),
            "without_router_first_seed": no_router, "overload_circular": stress, "routing": routing,
            "results_checked_against_alone": checked,
            "qps": runs["circular"][0]["qps"], "p50_ms": runs["circular"][0]["p50_ms"],
            "p99_ms": max(p99("circular"))}


def summary_of(per_query, batched, planner, serving) -> dict:
    """The headline figure of each section, so that the end of the line carries them all."""
    out = {"filter_aggregate_6M_frac_of_hbm": per_query["filter_aggregate_6M"].get("frac_of_hbm"),
           "query_a_frac_of_hbm": per_query["A"]["frac_of_hbm"], "query_b_frac_of_hbm": per_query["B"]["frac_of_hbm"]}
    if batched:
        out["batched_256_ms"] = batched["batched_ms"]
        out["batched_vs_one_at_a_time"] = batched["speedup"]
        out["batched_results_equal"] = batched["results_equal_one_at_a_time"]
    if planner and "plain_analytic_ms" in planner:
        out["config3_queries"] = planner["queries"]
        for k in ("plain_analytic_ms", "plain_learned_ms", "batched_analytic_ms", "batched_learned_ms",
                  "batched_analytic_one_window_ms", "batched_learned_one_window_ms",
                  "speedup_batched_learned_vs_plain_analytic", "speedup_batched_learned_one_window_vs_plain_analytic",
                  "results_identical_all_forms"):
            out["config3_" + k] = planner[k]
        live = planner["prediction_mae_live"]
        out["config3_mae_log_ms_learned"] = live["learned"]["mae_log_ms"]
        out["config3_mae_log_ms_analytic"] = live["analytic"]["mae_log_ms"]
    if serving:
        out["serving_qps"] = serving.get("qps")
        out["serving_p50_ms"] = serving.get("p50_ms")
        out["serving_p99_ms"] = serving.get("p99_ms")
    return out


def workload_config(n, s, world):
    """The `config` object both arms print: the workload named by what it is."""
    return {"workload": f"star join + group-by: Query A (category=1, region=1, group year x brand "
                        f"7x1000) + Query B (c_region=1, s_region=1, mfgr in {{0,1}}, group year x "
                        f"c_nation 7x25) over {n:,} fact rows per GPU",
            "fact_rows_per_gpu": n, "dims": {"supplier": s.s_len, "customer": s.c_len,
                                             "part": s.p_len, "date": s.d_len},
            "l2": f"{n * 16 / 1e9:.2f} GB + {n * 24 / 1e9:.2f} GB of fact columns per step"
                  + (", larger than the 126 MB L2, no flush" if n * 16 > 126e6 else ", within L2"),
            "parallelism": f"row shards x{world}", "seed": SEED}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    from mordred_b200 import ssb
    from oracle import oracle as O

    rows = min(args.rows, args.cpu_sample_rows * 5)
    trials = args.warmup + args.steps
    if O.ref_available(21) and O.ref_available(41):
        steps, cores = cpu_baseline_reference(rows, trials)
        kind = "reference"
    else:
        steps, cores = cpu_baseline_port(rows, trials)
        kind = "port"
    timed = steps[args.warmup:]
    ms = statistics.mean(timed)
    value = 2 * rows / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32 (int64 sums)", "data": "synthetic",
        "config": dict(workload_config(rows, ssb.Sizes(lo_len=rows), 1),
                       executed_on="host CPU: the reference's own engine, src/cpu/ssb/q21.cpp + q41.cpp"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{rows:,} fact rows per query, {args.steps} timed trials"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    from mordred_b200 import _lib as L
    from mordred_b200 import shard, ssb

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    L.call("mb_init", local)
    n = args.rows
    s = ssb.Sizes(lo_len=n)
    dims = sorted(set(ssb.QA_DIMS + ssb.QB_DIMS))
    # rank r holds rows [r*n, (r+1)*n) of one fact table; dimensions are replicated
    t = shard.gen_shard(s, SEED, ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"], rank, n)
    t.update(ssb.gen_device(s, SEED, [], dims))
    ws = ssb.StarWorkspace(s)
    dense = torch.zeros(ssb.QA_GROUPS + ssb.QB_GROUPS, dtype=torch.int64, device="cuda")

    def combine():
        # the only exchange: dense group sums of both queries, summed over ranks
        shard.allreduce_sums([shard.crystal4_sums(ws["res_a"]), shard.crystal4_sums(ws["res_b"])], dense)

    # per-step events around each probe launch, on the stream the kernels run on
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]

    def step(ev):
        cur = torch.cuda.current_stream()
        ssb.build_a(t, ws)
        if ev:
            ev[0].record(cur)
        ssb.probe_a(t, ws)
        if ev:
            ev[1].record(cur)
        ssb.build_b(t, ws)
        if ev:
            ev[2].record(cur)
        ssb.probe_b(t, ws)
        if ev:
            ev[3].record(cur)
        if world > 1:
            combine()

    for _ in range(args.warmup):
        step(None)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.launch_count()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record()
        for k in range(args.steps):
            step(evs[k])
        stop.record()
        torch.cuda.synchronize()
    launches = L.launch_count() - launches0
    probe_ms = {"A": [e[0].elapsed_time(e[1]) for e in evs], "B": [e[2].elapsed_time(e[3]) for e in evs]}
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    elapsed_ms = start.elapsed_time(stop)
    tmax = torch.tensor([elapsed_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    elapsed_ms = float(tmax.item())
    ms_step = elapsed_ms / args.steps
    rows_total = 2 * n * world * args.steps
    value = rows_total / (elapsed_ms / 1e3)
    status = L.device_status(local)

    # ---- roofline of the dominant kernel (the Query B probe: 24 B/row) ---------------------
    peak, peak_kind = measured_peaks()
    pa, pb = statistics.median(probe_ms["A"]), statistics.median(probe_ms["B"])
    dom = "B" if pb >= pa else "A"
    bytes_dom = n * (QB_BYTES_PER_ROW if dom == "B" else QA_BYTES_PER_ROW)
    achieved = bytes_dom / (pb if dom == "B" else pa) / 1e6  # bytes per ms -> GB/s
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        k = tj.get("q41_probe" if dom == "B" else "q21_probe")
        if k:
            traffic = k["bytes_per_launch_scaled"]

    # ---- filter-aggregate (16 B/row) on the full table, and on config 1's own 6 M-row table:
    # 20 separate 6 M-row copies (1.92 GB, far above L2) launched back to back from a CUDA
    # graph, so every launch reads its table from HBM with no flush inside the timed
    # region; per-launch time = replay time / 20. The old cold single launch (a 512 MB write
    # and a 512 MB read of other buffers before it) is reported beside it --------------------
    f_full = filter_aggregate_full(t, n, ws)
    f_small = filter_aggregate_6m(s, rank, peak)

    # ---- batched multi-query execution: 256 queries over the same fact rows ---------------
    batched = None if args.no_batch else batch_section(t, s, n, rank, world, args)

    # ---- end to end: host-resident tables through the public API ---------------------------
    e2e = None
    if not args.no_e2e:
        del t
        torch.cuda.empty_cache()
        h = ssb.gen_host(s, SEED + rank, ssb.QB_FACT, dims)
        runner = ssb.HostStarRunner(h, s)
        del h
        for _ in range(max(1, args.warmup // 2)):
            runner.run()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_steps = max(3, args.steps // 4)
        e0.record()
        for _ in range(e_steps):
            runner.run()
        e1.record()
        torch.cuda.synchronize()
        ems = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(ems, op=dist.ReduceOp.MAX)
        e_ms = float(ems.item()) / e_steps
        e2e = {"value": 2 * n * world * e_steps / (float(ems.item()) / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": runner.h2d_bytes, "d2h_bytes_per_step": runner.d2h_bytes,
               "ms_per_step": e_ms, "steps": e_steps,
               "h2d_gbs": runner.h2d_bytes / e_ms / 1e6,
               "bound": "host-to-device copies (PCIe Gen5 x16, 64 GB/s nominal per direction)"}

    # ---- config 3 (planner, host-resident table) and config 5 (serving) share one date-sorted
    # 600 M-row table in pinned host memory (N = 1) --------------------------------------------
    planner = serving = None
    table = None
    if world == 1 and (not args.no_planner or not args.no_serve):
        from mordred_b200.engine import SegmentedTable
        torch.cuda.empty_cache()
        table = SegmentedTable(args.planner_rows, SEED)
    if world == 1 and not args.no_planner:
        planner = planner_section(args, table)
    if world == 1 and not args.no_serve:
        torch.cuda.empty_cache()
        serving = serve_section(args, table)
    del table

    # ---- CPU baseline on the host cores (rank 0, N = 1) -------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        rows = args.cpu_sample_rows
        if O.ref_available(21) and O.ref_available(41):
            steps, cores = cpu_baseline_reference(rows, 3)
            kind = "reference"
        else:
            steps, cores = cpu_baseline_port(rows, 3)
            kind = "port"
        cms = min(steps[1:]) if len(steps) > 1 else steps[0]
        cpu = {"value": 2 * rows / (cms / 1e3), "unit": UNIT, "cores": cores, "kind": kind,
               "sample": f"Query A + Query B over {rows:,} of the {n:,} fact rows, best of 2 after 1 warm-up",
               "ms_per_step": cms}

    if rank == 0:
        per_query = {
            "filter_aggregate_6M": f_small,
            "filter_aggregate": {"ms": f_full, "fact_rows_per_s": n / (f_full / 1e3),
                                 "gbs": n * 16 / f_full / 1e6, "frac_of_hbm": n * 16 / f_full / 1e6 / peak},
            "A": {"probe_ms": pa, "fact_rows_per_s": n / (pa / 1e3), "gbs": n * QA_BYTES_PER_ROW / pa / 1e6,
                  "frac_of_hbm": n * QA_BYTES_PER_ROW / pa / 1e6 / peak},
            "B": {"probe_ms": pb, "fact_rows_per_s": n / (pb / 1e3), "gbs": n * QB_BYTES_PER_ROW / pb / 1e6,
                  "frac_of_hbm": n * QB_BYTES_PER_ROW / pb / 1e6 / peak},
        }
        # the long sections first; the line ends with the headline figures of every section
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32 (int64 sums)", "data": "synthetic",
            "config": workload_config(n, s, world),
            "planner": planner if world == 1 else {"skipped": "the planner experiment runs at N = 1"},
            "serving": serving if world == 1 else {"skipped": "the serving loop runs at N = 1"},
            "batched": batched,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "device_status": status,
            "roofline": {"bound": "hbm", "kernel": f"star_kernel (Query {dom} probe)", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bytes_dom},
            "per_query": per_query,
            "summary": summary_of(per_query, batched, planner if world == 1 else None,
                                  serving if world == 1 else None),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
