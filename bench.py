"""Benchmark: star join + group-by (Query A and Query B) over a 120,000,000-row fact table.

One step = Query A (3 filtered PHT builds + the fused supplier->part->date probe with
the 7x1000 group-by) and Query B (4 builds + the fused 4-way probe with the 7x25
group-by), each over every fact row. value = fact rows processed per second
(2 x 120 M per step per GPU). Inputs are synthetic (seeded generator with the
configured shapes) and larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

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
import subprocess
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
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


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


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
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
        "config": {"workload": f"Query A + Query B over {rows:,} fact rows on the host CPU "
                               "(src/cpu/ssb/q21.cpp + q41.cpp)", "fact_rows": rows},
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
    from mordred_b200 import ssb

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    L.call("mb_init", local)
    n = args.rows
    s = ssb.Sizes(lo_len=n)
    dims = sorted(set(ssb.QA_DIMS + ssb.QB_DIMS))
    # rank r holds rows [r*n, (r+1)*n) of one fact table; dimensions are replicated
    t = {}
    st = ssb._stream()
    for name in ssb.QB_FACT:
        buf = torch.empty(n, dtype=torch.int32, device="cuda")
        L.call("mb_gen_fact_column", ssb.FACT_COLUMNS[name], SEED, rank * n, n, s.s_len, s.c_len, s.p_len,
               ssb._p(buf), st)
        t[name] = buf
    t.update(ssb.gen_device(s, SEED, [], dims))
    ws = ssb.StarWorkspace(s)
    dense = torch.zeros(ssb.QA_GROUPS + ssb.QB_GROUPS, dtype=torch.int64, device="cuda")

    def combine():
        # the only exchange: dense group sums of both queries, summed over ranks
        ra = ws["res_a"].view(-1, 4)[:, 2:4].contiguous().view(torch.int64).view(-1)
        rb = ws["res_b"].view(-1, 4)[:, 2:4].contiguous().view(torch.int64).view(-1)
        dense[: ssb.QA_GROUPS].copy_(ra)
        dense[ssb.QA_GROUPS:].copy_(rb)
        dist.all_reduce(dense)

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
        e2e = {"value": 2 * n * world * e_steps / (float(ems.item()) / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": runner.h2d_bytes, "d2h_bytes_per_step": runner.d2h_bytes,
               "ms_per_step": float(ems.item()) / e_steps, "steps": e_steps}

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
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32 (int64 sums)", "data": "synthetic",
            "config": {"workload": f"star join + group-by: Query A (category=1, region=1, group year x brand "
                                   f"7x1000) + Query B (c_region=1, s_region=1, mfgr in {{0,1}}, group year x "
                                   f"c_nation 7x25) over {n:,} fact rows per GPU",
                       "fact_rows_per_gpu": n, "dims": {"supplier": s.s_len, "customer": s.c_len,
                                                        "part": s.p_len, "date": s.d_len},
                       "l2": "inputs larger than L2 (1.92 GB + 2.88 GB per step), no flush",
                       "parallelism": f"row shards x{world}", "seed": SEED},
            "per_query": {
                "A": {"probe_ms": pa, "fact_rows_per_s": n / (pa / 1e3), "gbs": n * QA_BYTES_PER_ROW / pa / 1e6,
                      "frac_of_hbm": n * QA_BYTES_PER_ROW / pa / 1e6 / peak},
                "B": {"probe_ms": pb, "fact_rows_per_s": n / (pb / 1e3), "gbs": n * QB_BYTES_PER_ROW / pb / 1e6,
                      "frac_of_hbm": n * QB_BYTES_PER_ROW / pb / 1e6 / peak},
            },
            "roofline": {"bound": "hbm", "kernel": f"star_kernel (Query {dom} probe)", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes_per_launch": bytes_dom},
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "device_status": status,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
