"""Autotuner for the fused star kernel.

For each query shape of the workload (the filter-aggregate, Query A, Query B and the
engine's four-table group-by) it times every launch configuration — consumer threads
per CTA, fact rows per thread, bulk-copy stages, shared-memory or L2 group
accumulation — on the current GPU with CUDA events, and writes the winners to
``mordred_b200/csrc/tuned_configs.h`` (the launcher's defaults, compiled into the
library) and the full measurements to ``mordred_b200/tuned_configs.json``.

    python -m mordred_b200.autotune [--rows N] [--write]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os

import torch

from . import _lib as L
from . import ssb

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "csrc", "tuned_configs.h")
JSON = os.path.join(HERE, "tuned_configs.json")

THREADS = (128, 256, 512)
WIDE_THREADS = (640, 768)  # 20 and 24 consumer warps over 16 tile slices (packed shapes only)
ITEMS = (4, 8, 16)
STAGES = (2, 3, 4, 6)


def _time(fn, reps: int = 5) -> float:
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def workload_shapes(n: int, seed: int = 1):
    """(name, bytes per row, key, args factory) for the tuned shapes."""
    s = ssb.Sizes(lo_len=n)
    t = ssb.gen_device(s, seed, ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"],
                       sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    ssb.build_a(t, ws)
    ht_c = torch.zeros(2 * s.c_len, dtype=torch.int32, device="cuda")
    ht_pb = torch.zeros(s.p_len, dtype=torch.int32, device="cuda")
    st = ssb._stream()
    L.call("mb_build_pht", ssb._p(t["c_region"]), 0, 1, 0, ssb._p(t["c_custkey"]), ssb._p(t["c_nation"]), s.c_len,
           ssb._p(ht_c), s.c_len, 0, None, st)
    L.call("mb_build_pht", ssb._p(t["p_mfgr"]), 2, 0, 1, ssb._p(t["p_partkey"]), None, s.p_len, ssb._p(ht_pb),
           s.p_len, 0, None, st)
    # engine layout tables for the four-table group-by
    eng = {}
    for name, key, val, flt, mode, c1, c2, slots, kmin in [
        ("s", "s_suppkey", None, "s_region", 1, 1, 1, s.s_len, 0),
        ("c", "c_custkey", "c_nation", "c_region", 1, 1, 1, s.c_len, 0),
        ("p", "p_partkey", None, "p_mfgr", 2, 0, 1, s.p_len, 0),
        ("d", "d_datekey", "d_year", None, 0, 0, 0, ssb.DATE_SLOTS, 19920101)]:
        ht = torch.zeros(2 * slots, dtype=torch.int32, device="cuda")
        import ctypes as C
        f = L.MbFilterArgsGPU(ssb._p(t[flt]) if flt else None, None, c1, c2, 0, 0, mode, 0)
        b = L.MbBuildArgsGPU(ssb._p(t[key]), ssb._p(t[val]) if val else None, slots, kmin, 0)
        L.call("mb_build_GPU2", None, C.byref(f), C.byref(b), s.dim_len(key), ssb._p(ht), 0, None, st)
        eng[name] = (ht, slots, kmin)
    res = torch.zeros(6 * 7000, dtype=torch.int32, device="cuda")
    big = 2**31

    def q11(**kw):
        return ssb.star_args(num_rows=n, filters=[dict(col=t["lo_discount"], c1=1, c2=3),
                                                  dict(col=t["lo_quantity"], c1=-big, c2=24),
                                                  dict(col=t["lo_orderdate"], c1=19930001, c2=19939999)],
                             aggr=[t["lo_extendedprice"], t["lo_discount"]], agg_op=L.MB_AGG_MUL,
                             res_layout=L.MB_RES_SCALAR, res=res, **kw)

    def qa(**kw):
        return ssb.star_args(num_rows=n, probes=[
            dict(fkey=t["lo_suppkey"], ht=ws["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_partkey"], ht=ws["ht_p_a"], num_slots=s.p_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
                 res_slot=1),
            dict(fkey=t["lo_orderdate"], ht=ws["ht_d"], num_slots=ssb.DATE_SLOTS, key_min=19920101,
                 layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)],
            aggr=[t["lo_revenue"]], agg_op=L.MB_AGG_SUM, total_val=ssb.QA_GROUPS, res_layout=L.MB_RES_CRYSTAL4,
            res=res, **kw)

    def qb(**kw):
        return ssb.star_args(num_rows=n, probes=[
            dict(fkey=t["lo_suppkey"], ht=ws["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_custkey"], ht=ht_c, num_slots=s.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7, res_slot=1),
            dict(fkey=t["lo_partkey"], ht=ht_pb, num_slots=s.p_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_orderdate"], ht=ws["ht_d"], num_slots=ssb.DATE_SLOTS, key_min=19920101,
                 layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)],
            aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=ssb.QB_GROUPS,
            res_layout=L.MB_RES_CRYSTAL4, res=res, **kw)

    def engine(**kw):
        probes = []
        for slot, (k, fk, mn, uq) in enumerate([("s", "lo_suppkey", 0, 0), ("c", "lo_custkey", 0, 7),
                                                 ("p", "lo_partkey", 0, 0), ("d", "lo_orderdate", 1992, 1)]):
            ht, slots, kmin = eng[k]
            probes.append(dict(fkey=t[fk], ht=ht, num_slots=slots, key_min=kmin, layout=L.MB_HT_VAL_OFF,
                               min_val=mn, unique_val=uq, res_slot=slot))
        return ssb.star_args(num_rows=n, probes=probes, aggr=[t["lo_revenue"], t["lo_supplycost"]],
                             agg_op=L.MB_AGG_SUB, total_val=ssb.QB_GROUPS, res_layout=L.MB_RES_ENGINE6, res=res, **kw)

    return [
        ("filter-aggregate (q11 form)", 16, (3, 0, -1, 0, 0), q11),
        ("Query A form", 16, (0, 3, 0, 1, 1), qa),
        ("Query B form", 24, (0, 4, 0, 1, 0), qb),
        ("engine four-table group-by", 24, (0, 4, 2, 1, 0), engine),
    ], (t, ws, ht_c, ht_pb, eng, res)


def tune(n: int = 120_000_000, reps: int = 5, verbose: bool = True) -> list[dict]:
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    shapes, keep = workload_shapes(n)
    results = []
    for name, bpr, key, make in shapes:
        runs = []
        packed, early = tuple(key) in PACKED_SHAPES, tuple(key) in EARLY_RETURN_SHAPES
        threads = THREADS + (WIDE_THREADS if packed or early else ())
        # mb_star_args.pack: 1 plain, 2 packed, 3 packed with early stage return, 4 unpacked
        # with early stage return
        packs = (1, 2, 3) if packed else (1, 4) if early else (1,)
        for th, it, stg, gm, pk in itertools.product(threads, ITEMS, STAGES, (1, 2), packs):
            if key[3] == 0 and gm == 2:
                continue  # scalar results have no group array
            try:
                a = make(threads=th, items_per_thread=it, stages=stg, group_mode=gm if key[3] else 0, pack=pk)
                ms = _time(lambda: ssb.star_query(a), reps)
            except L.MbError:
                continue
            runs.append({"threads": th, "items": it, "stages": stg, "group_mode": gm if key[3] else 0,
                         "pack": pk - 1, "ms": ms})
        runs.sort(key=lambda r: r["ms"])
        best = runs[0]
        gbs = n * bpr / best["ms"] / 1e6
        if verbose:
            print(f"{name}: best {best} -> {gbs:.0f} GB/s", flush=True)
        results.append({"shape": name, "key": list(key), "bytes_per_row": bpr, "rows": n, "best": best,
                        "gbs": gbs, "runs": runs})
    if L.device_status(0) != 0:
        raise RuntimeError("device status set during tuning")
    return results


def tune_small(n: int = 6_000_000, copies: int = 20, reps: int = 10, verbose: bool = True) -> dict:
    """The filter-aggregate on tables of n rows (fit in L2 on their own): `copies` separate
    tables launched back to back from a CUDA graph, so every launch reads its table from
    HBM; per-launch time = replay time / copies. Also sweeps the grid (CTAs)."""
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    s = ssb.Sizes(lo_len=n)
    tabs = [ssb.gen_device(s, 9000 + k, ssb.Q11_COLUMNS, []) for k in range(copies)]
    rev = torch.zeros(copies, dtype=torch.int64, device="cuda")
    big = 2**31

    def args(k, **kw):
        t = tabs[k]
        return ssb.star_args(num_rows=n, filters=[dict(col=t["lo_discount"], c1=1, c2=3),
                                                  dict(col=t["lo_quantity"], c1=-big, c2=24),
                                                  dict(col=t["lo_orderdate"], c1=19930001, c2=19939999)],
                             aggr=[t["lo_extendedprice"], t["lo_discount"]], agg_op=L.MB_AGG_MUL,
                             res_layout=L.MB_RES_SCALAR, res=rev[k:], **kw)

    runs = []
    for th, it, stg, grid in itertools.product(THREADS, ITEMS, STAGES, (0, 148, 296, 444)):
        try:
            al = [args(k, threads=th, items_per_thread=it, stages=stg, grid=grid) for k in range(copies)]
            for a in al:
                ssb.star_query(a)
        except L.MbError:
            continue
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for a in al:
                ssb.star_query(a)
        ms = _time(g.replay, reps) / copies
        del g
        runs.append({"threads": th, "items": it, "stages": stg, "grid": grid, "group_mode": 0, "ms": ms})
    runs.sort(key=lambda r: r["ms"])
    best = [r for r in runs if r["grid"] == 0][0]  # the header carries no grid: the launcher's own
    gbs = n * 16 / best["ms"] / 1e6
    if verbose:
        print(f"filter-aggregate, {n:,} rows: best {best} -> {gbs:.0f} GB/s", flush=True)
    if L.device_status(0) != 0:
        raise RuntimeError("device status set during tuning")
    return {"shape": f"filter-aggregate, {n // 1_000_000} M rows", "key": [3, 0, -1, 0, 0], "bytes_per_row": 16,
            "rows": n, "max_rows": 16 << 20, "best": best, "gbs": gbs, "runs": runs}


# Shapes whose sparse phase runs the packed second round (star_kernel<..., PACK = true>),
# measured at 120 M rows: the Query B shape 0.686 against 0.710 ms, the engine four-table
# shape (customer probed first, the supplier read for its payload afterwards) 0.754
# against 0.808 ms; the Query A shape has no packed variant (its second round is one
# small table, and packing cost more than it saved: 0.565 against 0.460 ms). These shapes
# also have the variants that return each stage before the last batch's probes
# (REL = true) and run 20 or 24 consumer warps over 16 tile slices: Query B 0.627 against
# 0.724 ms, the engine shape 0.666 against 0.795 ms for the 16-warp packed kernel (same
# box); returning the stage after the last batch's first probe round instead, with only
# the kept rows copied, measured 0.638 / 0.674 ms against 0.611 / 0.653 ms. The tuned
# entry's pack field: 1 packed, 2 packed with early stage return.
PACKED_SHAPES = {(0, 4, 0, 1, 0), (0, 4, 2, 1, 0)}
# Shapes with unpacked early-return variants (20 or 24 consumer warps): Query A, 0.4526
# against 0.460 ms for three 8-warp CTAs a SM (it already had 24 consumer warps a SM).
EARLY_RETURN_SHAPES = {(0, 3, 0, 1, 1)}


def write(results: list[dict], gpu: str) -> None:
    lines = []
    for r in sorted(results, key=lambda r: -r.get("max_rows", 0)):  # row-limited entries first
        b, k = r["best"], r["key"]
        limit = f", {r['max_rows'] >> 20}ll << 20" if r.get("max_rows") else ""
        pack = f", 0, {b['pack']}" if b.get("pack") else ""
        lines.append(f"    {{{k[0]}, {k[1]}, {k[2]}, {k[3]}, {k[4]}, {{{b['threads']}, {b['items']}, {b['stages']}, "
                     f"{b['group_mode']}{pack}}}{limit}}},  // {r['shape']}: {b['ms']:.4f} ms, {r['gbs'] / 1000:.2f} TB/s")
    text = open(HEADER).read()
    head, rest = text.split("static const TunedEntry kTuned[] = {\n", 1)
    _, tail = rest.split("};\n", 1)
    open(HEADER, "w").write(head + "static const TunedEntry kTuned[] = {\n" + "\n".join(lines) + "\n};\n" + tail)
    json.dump({"gpu": gpu, "results": results}, open(JSON, "w"), indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=120_000_000)
    ap.add_argument("--write", action="store_true")
    args = ap.parse_args()
    res = tune(args.rows) + [tune_small()]
    if args.write:
        write(res, torch.cuda.get_device_name(0))


if __name__ == "__main__":
    main()
