"""The learned-planner experiment: log per-segment timings, train the cost MLP, and
compare it with the analytic cost model on prediction error and on end-to-end query
time over a host-resident fact table with a GPU segment cache.

    python -m mordred_b200.planner_experiment [--rows 600000000] [--log-samples 50000]
        [--eval-queries 300] [--save mordred_b200/planner_weights/mlp.bin] [--out FILE]
        [--weights FILE]   # evaluate saved weights instead of logging and training

Workload: queries from the seeded generator over the filter-aggregate, Query A and
Query B forms, selectivities log-uniform in [1e-5, 0.3] (different seeds for the
training log and the evaluation). The table is sorted by orderdate, so a query's date
range skips whole segments. The GPU segment cache holds `--cache-gb` of the table's
column segments (8 GB = 2,048 segments of 4 MiB by default).

Logging: per training query, up to --per-query segments are timed on each device, alone
and together (Executor.profile_segments: a segment's cost is its share of the batched
time plus its own admission copies), and the query's hash-table builds on each device
are timed as its fixed costs; every --shuffle-every queries the cache is refilled at
random so that the log covers every residency. Evaluation: both planners run the same
evaluation queries from the same starting cache (the segments of the most used columns,
as an epoch replacement by column frequency would leave it); results must agree bit for
bit; the JSON reports per-planner total / p50 / p99 ms and the MAE of each model's log
predictions on held-out logged segments.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import time

import numpy as np
import torch

from . import _lib as L
from . import batch as B
from .engine import COL_ID, FACT, NEEDED, SEG, Executor, SegmentedTable
from .planner import MIN_MS, AnalyticPlanner, LearnedPlanner

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "planner_weights", "mlp.bin")


def initial_weights(t: SegmentedTable, queries: list[B.Query]) -> np.ndarray:
    """Epoch-replacement weights: each column's segments weighted by how many queries of
    the workload read the column (CacheManager.cu:534-588 fills the cache heaviest first)."""
    w = np.zeros((len(FACT), t.nseg))
    for q in queries:
        for c in NEEDED[q.template]:
            w[COL_ID[c]] += 1.0
    # earlier segments first within a column, so the fill is deterministic
    w += np.linspace(1e-3, 0, t.nseg)[None, :]
    return w


def refill(ex: Executor, weights: np.ndarray) -> None:
    ex.cache.replace(weights, [ex.t.ptr(c, 0) for c in FACT], ex.t.seg_rows)
    torch.cuda.synchronize()


def collect_log(ex: Executor, n_samples: int, seed: int, per_query: int, shuffle_every: int, log=print) -> dict:
    rng = np.random.default_rng(seed)
    qs_seed = seed
    recs = []
    fixed = []
    nq = 0
    t0 = time.perf_counter()
    while len(recs) < n_samples:
        for q in B.generate_queries(200, seed=qs_seed):
            if len(recs) >= n_samples:
                break
            if nq % shuffle_every == 0:
                # a random residency: random positive weights on a random share of the segments
                w = rng.random((len(FACT), ex.t.nseg)) * (rng.random((len(FACT), ex.t.nseg)) < rng.uniform(0.1, 1))
                refill(ex, w)
            nq += 1
            cand = ex.candidates(q)
            if len(cand) == 0:
                continue
            pick = rng.choice(cand, min(per_query, len(cand)), replace=False)
            r, f = ex.profile_segments(q, pick)
            recs += r
            fixed.append(f)
        qs_seed += 1
        log(f"  logged {len(recs)} segment timings from {nq} queries, {time.perf_counter() - t0:.0f} s")
    recs = recs[:n_samples]
    return {"features": np.stack([r["features"] for r in recs]).astype(np.float32),
            "log_ms": np.log(np.maximum([[r["cpu_ms"], r["gpu_ms"]] for r in recs], MIN_MS)).astype(np.float32),
            "analytic_log_ms": np.log(np.maximum([[r["analytic_cpu_ms"], r["analytic_gpu_ms"]] for r in recs],
                                                 MIN_MS)).astype(np.float32),
            "solo_log_ms": np.log(np.maximum([[r["cpu_solo_ms"], r["gpu_solo_ms"]] for r in recs],
                                              MIN_MS)).astype(np.float32),
            "template": np.array([r["template"] for r in recs]), "queries": nq,
            "fixed_ms": {t: [float(np.median([f["cpu_build_ms"] for f in fixed if f["template"] == t] or [0.0])),
                             float(np.median([f["gpu_build_ms"] for f in fixed if f["template"] == t] or [0.0]))]
                         for t in ("agg", "qa", "qb")},
            "seconds": time.perf_counter() - t0}


def mae_report(pred: np.ndarray, truth: np.ndarray) -> dict:
    err = np.abs(pred - truth)
    return {"mae_log_cpu_ms": float(err[:, 0].mean()), "mae_log_gpu_ms": float(err[:, 1].mean()),
            "mae_log_ms": float(err.mean())}


def completion_stats(ms: list[float]) -> dict:
    """Latency of queries that all arrived at time 0 and ran in the given order: each one's
    completion time is the running total of the service times before and including it."""
    done = np.cumsum(ms)
    return {"p50_completion_ms": float(np.percentile(done, 50)), "p99_completion_ms": float(np.percentile(done, 99))}


def evaluate(ex: Executor, planners: list, queries: list[B.Query], start_weights: np.ndarray, log=print,
             keep_results: dict | None = None) -> dict:
    """Run `queries` one at a time under each planner from the same starting cache. When
    keep_results is a dict, each planner's per-query results are stored in it by name."""
    out = {}
    results = {}
    for p in planners:
        refill(ex, start_weights)
        # one untimed query loads the kernels and the pool threads
        ex.run(queries[0], p)
        refill(ex, start_weights)
        ms, gseg, cseg, adm = [], 0, 0, 0
        res = []
        diag = {"gpu_ms": 0.0, "cpu_ms": 0.0, "pred_gpu_ms": 0.0, "pred_cpu_ms": 0.0, "plan_ms": 0.0,
                "cpu_bound_queries": 0}
        for q in queries:
            r = ex.run(q, p)
            ms.append(r.ms)
            gseg += r.gpu_segments
            cseg += r.cpu_segments
            adm += r.admitted
            res.append(r.result)
            diag["gpu_ms"] += r.gpu_ms
            diag["cpu_ms"] += r.cpu_ms
            diag["cpu_bound_queries"] += int(r.cpu_ms > r.gpu_ms)
            for k in ("pred_gpu_ms", "pred_cpu_ms", "plan_ms"):
                diag[k] += r.extra.get(k, 0.0)
        results[p.name] = res
        if keep_results is not None:
            keep_results[p.name] = res
        ms_sorted = sorted(ms)
        out[p.name] = {"total_ms": float(sum(ms)), "mean_ms": float(statistics.mean(ms)),
                       "p50_ms": float(ms_sorted[len(ms) // 2]),
                       "p99_ms": float(ms_sorted[min(len(ms) - 1, int(math.ceil(0.99 * len(ms))) - 1)]),
                       **completion_stats(ms),
                       "gpu_segments": gseg, "cpu_segments": cseg, "column_segments_admitted": adm,
                       "sums": diag}
        log(f"  {p.name}: total {out[p.name]['total_ms']:.0f} ms over {len(queries)} queries, "
            f"p50 {out[p.name]['p50_ms']:.2f}, p99 {out[p.name]['p99_ms']:.2f}, gpu/cpu segments {gseg}/{cseg}")
    names = list(results)
    out["results_identical"] = all(np.array_equal(a, b) for a, b in zip(results[names[0]], results[names[-1]]))
    return out


def evaluate_batched(bx, planners: list, queries: list[B.Query], start_weights: np.ndarray, window: int = 256,
                     log=print, keep_results: dict | None = None) -> dict:
    """Run `queries` in windows of `window` through the batched executor under each planner,
    from the same starting cache (and no carried-over benefit weights)."""
    out = {}
    for p in planners:
        bx.benefit[:] = 0.0
        bx.cache.replace(start_weights, bx.host_ptrs, bx.t.seg_rows)
        bx.run_window(queries[:8], p)           # loads kernels, pool threads, model
        bx.benefit[:] = 0.0
        bx.cache.replace(start_weights, bx.host_ptrs, bx.t.seg_rows)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        runs = bx.run(queries, p, window=window)
        total = (time.perf_counter() - t0) * 1e3
        res = [r for w in runs for r in w.results]
        if keep_results is not None:
            keep_results[p.name] = res
        # windows overlap (the next is planned and enqueued while one runs): a query
        # completes when its window's results are merged
        done = np.array([(w.extra["done_at"] - t0) * 1e3 for w in runs])
        per_query = np.repeat(done, [w.queries for w in runs])
        out[p.name] = {"total_ms": total, "windows": len(runs), "window_queries": window,
                       "mean_window_ms": float(np.mean([w.ms for w in runs])),
                       "p50_completion_ms": float(np.percentile(per_query, 50)),
                       "p99_completion_ms": float(np.percentile(per_query, 99)),
                       "union_segments": int(sum(w.union_segments for w in runs)),
                       "gpu_segments": int(sum(w.gpu_segments for w in runs)),
                       "cpu_segments": int(sum(w.cpu_segments for w in runs)),
                       "staged_column_segments": int(sum(w.staged_segments for w in runs)),
                       "admitted_column_segments": int(sum(w.copied_column_segments for w in runs)),
                       "launches": int(sum(w.launches for w in runs)),
                       "plan_ms": float(sum(w.plan_ms for w in runs)), "gpu_ms": float(sum(w.gpu_ms for w in runs)),
                       "cpu_ms": float(sum(w.cpu_ms for w in runs))}
        log(f"  batched {p.name}: total {total:.0f} ms over {len(queries)} queries in {len(runs)} windows")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=600_000_000)
    ap.add_argument("--seed", type=int, default=20260101)
    ap.add_argument("--cache-gb", type=float, default=8.0)
    ap.add_argument("--log-samples", type=int, default=50_000)
    ap.add_argument("--per-query", type=int, default=32)
    ap.add_argument("--shuffle-every", type=int, default=25)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--eval-queries", type=int, default=300)
    ap.add_argument("--weights", default=None, help="evaluate these saved weights (skip logging and training)")
    ap.add_argument("--save", default=None)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    log = lambda *a: print(*a, flush=True)
    t0 = time.perf_counter()
    table = SegmentedTable(args.rows, args.seed)
    slots = int(args.cache_gb * (1 << 30) // (SEG * 4))
    ex = Executor(table, cache_slots=slots, policy="lru")
    log(f"table: {args.rows:,} rows, {table.nseg} segments x {len(FACT)} columns in pinned host memory; "
        f"cache {slots} slots; {time.perf_counter() - t0:.0f} s")
    report = {"rows": args.rows, "segments": table.nseg, "cache_slots": slots, "seed": args.seed,
              "cpu_threads": ex.cpu_threads}
    if args.weights:
        learned = LearnedPlanner.load(args.weights)
        report["weights"] = os.path.relpath(args.weights, os.path.dirname(HERE))
        report["training"] = learned.manifest.get("training", {})
        report["holdout"] = learned.manifest.get("holdout", {})
    else:
        data = collect_log(ex, args.log_samples, args.seed + 1, args.per_query, args.shuffle_every, log)
        n = len(data["features"])
        perm = np.random.default_rng(0).permutation(n)
        cut = int(0.9 * n)
        tr, ho = perm[:cut], perm[cut:]
        learned = LearnedPlanner(seed=0, fixed_ms=data["fixed_ms"])
        tt = time.perf_counter()
        learned.train(data["features"][tr], data["log_ms"][tr], epochs=args.epochs)
        train_s = time.perf_counter() - tt
        pred = learned.predict_log(data["features"][ho])
        holdout = {"samples": int(len(ho)), "learned": mae_report(pred, data["log_ms"][ho]),
                   "analytic": mae_report(data["analytic_log_ms"][ho], data["log_ms"][ho])}
        report["log"] = {"samples": n, "queries": data["queries"], "seconds": data["seconds"],
                         "by_template": {k: int((data["template"] == k).sum()) for k in ("agg", "qa", "qb")},
                         "median_cpu_ms": float(np.exp(np.median(data["log_ms"][:, 0]))),
                         "median_gpu_ms": float(np.exp(np.median(data["log_ms"][:, 1]))),
                         "median_cpu_solo_ms": float(np.exp(np.median(data["solo_log_ms"][:, 0]))),
                         "median_gpu_solo_ms": float(np.exp(np.median(data["solo_log_ms"][:, 1]))),
                         "fixed_ms": data["fixed_ms"]}
        report["training"] = dict(learned.record, seconds=train_s, train_loss_per_epoch=None,
                                  final_train_loss=learned.record["train_loss_per_epoch"][-1])
        report["holdout"] = holdout
        log(f"  hold-out MAE of log ms: learned {holdout['learned']['mae_log_ms']:.3f}, "
            f"analytic {holdout['analytic']['mae_log_ms']:.3f}")
        if args.save:
            learned.save(args.save, {"holdout": holdout, "log": report["log"], "rows": args.rows,
                                     "cache_slots": slots, "cpu_threads": ex.cpu_threads})
    queries = B.generate_queries(args.eval_queries, seed=args.seed + 7)
    start = initial_weights(table, queries)
    report["evaluation"] = evaluate(ex, [AnalyticPlanner(), learned], queries, start, log)
    ev = report["evaluation"]
    report["evaluation"]["speedup_learned_vs_analytic"] = ev["analytic"]["total_ms"] / ev["learned"]["total_ms"]
    report["device_status"] = L.device_status(0)
    report["seconds"] = time.perf_counter() - t0
    line = json.dumps(report)
    print(line, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
