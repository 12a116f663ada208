"""Run one of the library's kernels on a chosen table size a few times, for profilers.

    python -m mordred_b200.profile_case [--case NAME] [--rows N] [--reps K]

Cases (each through the C ABI, then a check of the device status word):
  ssb       filter-aggregate (mb_q11_query), Query A and Query B (builds + probes) with the
            tuned launch defaults (the default case)
  mirrors   Query A and Query B probes with cluster-resident mirrors forced on
  engine    the engine's probe_group_by over VAL_OFF tables, direct columns and through a
            segment cache (mb_probe_group_by_GPU2)
  select    selection with compaction (mb_filter_probe_GPU2: offset list + dimension rows)
  list      the offset-list group-by over that list (mb_probe_group_by_GPU3)
  build     the dimension builds (mb_build_pht, mb_build_GPU2) at full dimension sizes
  batch     a batch of --batch generated queries (mb_pat_build, mb_batch_run)
  noalloc   the Query B probe without allocation (mb_q41_probe_noalloc)
  mlp       the planner MLP: forward, backward and Adam over 50,000 samples
Small sizes (for example 24,000,000 rows: 576 MB of fact columns, above the 126 MB L2)
keep an ncu capture short.
"""
from __future__ import annotations

import argparse
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from . import ssb

SEG = 1 << 20


def _ssb(args, s):
    t = ssb.gen_device(s, args.seed, ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"],
                       sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    for _ in range(args.reps):
        ssb.q11(t, args.rows, ws)
        ssb.query_a(t, ws)
        ssb.query_b(t, ws)


def _mirrors(args, s):
    t = ssb.gen_device(s, args.seed, ssb.QB_FACT, sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    ssb.build_a(t, ws)
    ssb.build_b(t, ws)
    d = dict(num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN, layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1,
             res_slot=0)
    qa = ssb.star_args(num_rows=args.rows, probes=[
        dict(fkey=t["lo_suppkey"], ht=ws["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
        dict(fkey=t["lo_partkey"], ht=ws["ht_p_a"], num_slots=s.p_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
             res_slot=1), dict(fkey=t["lo_orderdate"], ht=ws["ht_d"], **d)],
        aggr=[t["lo_revenue"]], agg_op=L.MB_AGG_SUM, total_val=ssb.QA_GROUPS, res_layout=L.MB_RES_CRYSTAL4,
        res=ws["res_a"], mirrors=2)
    qb = ssb.star_args(num_rows=args.rows, probes=[
        dict(fkey=t["lo_suppkey"], ht=ws["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
        dict(fkey=t["lo_custkey"], ht=ws["ht_c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
             res_slot=1), dict(fkey=t["lo_partkey"], ht=ws["ht_p_b"], num_slots=s.p_len, layout=L.MB_HT_KEY),
        dict(fkey=t["lo_orderdate"], ht=ws["ht_d"], **d)],
        aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=ssb.QB_GROUPS,
        res_layout=L.MB_RES_CRYSTAL4, res=ws["res_b"], mirrors=2)
    for _ in range(args.reps):
        ssb.star_query(qa)
        ssb.star_query(qb)


def _engine_tables(s, t):
    """VAL_OFF (engine) tables of the four dimensions, built by mb_build_GPU2."""
    hts = {}
    for name, key, val, flt, mode, c1, c2, slots, kmin in [
            ("s", "s_suppkey", None, "s_region", 1, 1, 1, s.s_len, 0),
            ("c", "c_custkey", "c_nation", "c_region", 1, 1, 1, s.c_len, 0),
            ("p", "p_partkey", None, "p_mfgr", 2, 0, 1, s.p_len, 0),
            ("d", "d_datekey", "d_year", None, 0, 0, 0, ssb.DATE_SLOTS, ssb.DATE_MIN)]:
        ht = torch.zeros(2 * slots, dtype=torch.int32, device="cuda")
        f = L.MbFilterArgsGPU(ssb._p(t[flt]) if flt else None, None, c1, c2, 0, 0, mode, 0)
        b = L.MbBuildArgsGPU(ssb._p(t[key]), ssb._p(t[val]) if val else None, slots, kmin, 0)
        L.call("mb_build_GPU2", None, C.byref(f), C.byref(b), t[key].numel(), ssb._p(ht), 0, None, ssb._stream())
        hts[name] = (ht, slots, kmin)
    return hts


def _cache(t, names, n=None):
    """The named columns in one segment cache (consecutive slots per column)."""
    lens = {k: t[k].numel() if n is None else n for k in names}
    nslots = sum((lens[k] + SEG - 1) // SEG for k in names)
    pool = torch.zeros(nslots * SEG, dtype=torch.int32, device="cuda")
    idx, first = {}, 0
    for name in names:
        nseg = (lens[name] + SEG - 1) // SEG
        for sg in range(nseg):
            lo, hi = sg * SEG, min((sg + 1) * SEG, lens[name])
            pool[(first + sg) * SEG: (first + sg) * SEG + (hi - lo)] = t[name][lo:hi]
        idx[name] = torch.arange(first, first + nseg, dtype=torch.int32, device="cuda")
        first += nseg
    return pool, idx


def _engine(args, s):
    t = ssb.gen_device(s, args.seed, ssb.QB_FACT, ssb.QB_DIMS)
    hts = _engine_tables(s, t)
    names = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost"]
    pool, idx = _cache(t, names)
    g = L.MbGroupbyArgsGPU(None, None, None, None, None, None, 0, 0, 0, 1992, 0, 7, 0, 1, ssb.QB_GROUPS, 0)
    res = torch.zeros(6 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
    for cache in (False, True):
        cols = idx if cache else t
        p = L.MbProbeArgsGPU(*(ssb._p(cols[k]) for k in names[:4]), *(ssb._p(hts[k][0]) for k in "scpd"),
                             *(hts[k][1] for k in "scpd"), *(hts[k][2] for k in "scpd"))
        g.aggr_idx1, g.aggr_idx2 = ssb._p(cols["lo_revenue"]), ssb._p(cols["lo_supplycost"])
        for _ in range(args.reps):
            L.call("mb_probe_group_by_GPU2", ssb._p(pool) if cache else None, C.byref(p), C.byref(g), args.rows,
                   ssb._p(res), 0, None, ssb._stream())


def _select_and_list(args, s, do_list):
    t = ssb.gen_device(s, args.seed, ssb.QB_FACT, ssb.QB_DIMS)
    hts = _engine_tables(s, t)
    names = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost", "c_nation"]
    pool, idx = _cache(t, names)
    lo = torch.zeros(args.rows, dtype=torch.int32, device="cuda")
    dc = torch.zeros(args.rows, dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    f = L.MbFilterArgsGPU(ssb._p(idx["lo_orderdate"]), None, 19940101, 19961231, 0, 0, 1, 0)
    p = L.MbProbeArgsGPU(ssb._p(idx["lo_suppkey"]), ssb._p(idx["lo_custkey"]), None, None, ssb._p(hts["s"][0]),
                         ssb._p(hts["c"][0]), None, None, s.s_len, s.c_len, 0, 0, 0, 0, 0, 0)
    out = L.MbOffsetGPU(ssb._p(lo), None, ssb._p(dc), None, None)
    for _ in range(args.reps if not do_list else 1):
        total.zero_()
        L.call("mb_filter_probe_GPU2", ssb._p(pool), C.byref(f), C.byref(p), C.byref(out), args.rows, ssb._p(total),
               0, None, ssb._stream())
    if not do_list:
        return
    k = int(total.item())
    # the list form: probe part and date, group by (customer nation passed through at the
    # customer rows the selection recorded, year)
    pl = L.MbProbeArgsGPU(None, None, ssb._p(idx["lo_partkey"]), ssb._p(idx["lo_orderdate"]), None, None,
                          ssb._p(hts["p"][0]), ssb._p(hts["d"][0]), 0, 0, s.p_len, ssb.DATE_SLOTS, 0, 0, 0,
                          ssb.DATE_MIN)
    g = L.MbGroupbyArgsGPU(ssb._p(idx["lo_revenue"]), ssb._p(idx["lo_supplycost"]), None, ssb._p(idx["c_nation"]),
                           None, None, 0, 0, 0, 1992, 0, 7, 0, 1, ssb.QB_GROUPS, 0)
    res = torch.zeros(6 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
    off = L.MbOffsetGPU(ssb._p(lo), None, ssb._p(dc), None, None)
    for _ in range(args.reps):
        L.call("mb_probe_group_by_GPU3", ssb._p(pool), C.byref(off), C.byref(pl), C.byref(g), k, ssb._p(res),
               ssb._stream())


def _build(args, s):
    t = ssb.gen_device(s, args.seed, [], sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    for _ in range(args.reps):
        ssb.build_a(t, ws)
        ssb.build_b(t, ws)
        _engine_tables(s, t)


def _batch(args, s):
    from . import batch as B
    t = ssb.gen_device(s, args.seed, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    qs = B.generate_queries(args.batch or 256, seed=args.seed)
    res = [q.result_buffer() for q in qs]
    for _ in range(args.reps):
        B.run_batch(t, pats, qs, res, args.rows)


def _noalloc(args, s):
    t = ssb.gen_device(s, args.seed, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    ssb.build_b(t, ws)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(args.reps):
        L.call("mb_q41_probe_noalloc", *[ssb._p(t[k]) for k in ("lo_orderdate", "lo_partkey", "lo_custkey",
                                                                  "lo_suppkey", "lo_revenue", "lo_supplycost")],
               s.lo_len, ssb._p(ws["ht_p_b"]), s.p_len, ssb._p(ws["ht_s"]), s.s_len, ssb._p(ws["ht_c"]), s.c_len,
               ssb._p(ws["ht_d"]), ssb.DATE_SLOTS, ssb._p(ws["res_b"]), ssb._p(status), ssb._stream())


def _mlp(args, s):
    from .planner import LearnedPlanner
    rng = np.random.default_rng(args.seed)
    n = 50_000
    feats = rng.normal(size=(n, L.MB_MLP_IN)).astype(np.float32)
    target = rng.normal(size=(n, 2)).astype(np.float32)
    pl = LearnedPlanner(seed=args.seed)
    pl.train(feats, target, epochs=args.reps)
    pl.predict_log(feats)


CASES = {"ssb": _ssb, "mirrors": _mirrors, "engine": _engine, "select": lambda a, s: _select_and_list(a, s, False),
         "list": lambda a, s: _select_and_list(a, s, True), "build": _build, "batch": _batch, "noalloc": _noalloc,
         "mlp": _mlp}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="ssb", choices=sorted(CASES))
    ap.add_argument("--rows", type=int, default=24_000_000)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--batch", type=int, default=0, help="batch case: this many generated queries (256)")
    args = ap.parse_args()
    if args.batch and args.case == "ssb":
        args.case = "batch"
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    s = ssb.Sizes(lo_len=args.rows)
    CASES[args.case](args, s)
    torch.cuda.synchronize()
    st = L.device_status(0)
    if st:
        raise SystemExit(f"device status {st:#x}")
    print(f"ok: case {args.case}, {args.reps} reps over {args.rows:,} rows; {L.launch_count()} library launches")


if __name__ == "__main__":
    main()
