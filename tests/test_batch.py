"""Batched multi-query execution: the workload generator (CPU) and, on the GPU, every
query of a batch against the same query run alone (bit for bit) and against the oracle."""
import numpy as np
import pytest

from mordred_b200 import batch as B
from mordred_b200 import ssb


def test_generator_is_seeded_and_spans_selectivities():
    a = B.generate_queries(300, seed=7)
    b = B.generate_queries(300, seed=7)
    assert [(q.template, q.date, q.s_region, q.category) for q in a] == \
           [(q.template, q.date, q.s_region, q.category) for q in b]
    assert {q.template for q in a} == {"agg", "qa", "qb"}
    sels = np.array([q.meta["expected_selectivity"] for q in a])
    assert sels.min() < 1e-3 and sels.max() > 0.05
    for q in a:
        assert q.date[0] <= q.date[1] and q.date[0] in B.CALENDAR and q.date[1] in B.CALENDAR
        assert 0 <= q.s_region[0] <= q.s_region[1] <= 4 and 0 <= q.category[0] <= q.category[1] <= 24
        assert 1 <= q.quantity[0] <= q.quantity[1] <= 50 and 0 <= q.discount[0] <= q.discount[1] <= 10
    assert {q.groups for q in a} == {1, 175, 7000}


def test_descriptor_fields_fit_the_encoding():
    for q in B.generate_queries(30, seed=1):
        c = q.to_c(type("R", (), {"data_ptr": lambda self: 4096})())
        assert 1 <= c.num_preds <= 4
        for i in range(c.num_preds):
            assert 0 <= c.pred_field[i] < 65536 and c.pred_lo[i] <= c.pred_hi[i]


@pytest.mark.gpu
@pytest.mark.parametrize("n_rows,n_queries", [(1_000_003, 40), (4_194_304, 96)])
def test_batch_equals_alone(n_rows, n_queries):
    import torch
    from mordred_b200 import _lib as L
    torch.cuda.set_device(0)
    s = ssb.Sizes(lo_len=n_rows, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(s, 314, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    qs = B.generate_queries(n_queries, seed=n_queries, sel_lo=1e-4, sel_hi=0.5)
    res_b = [q.result_buffer() for q in qs]
    B.run_batch(t, pats, qs, res_b, n_rows)
    ws = B.AloneWorkspace(s)
    for i, q in enumerate(qs):
        r = q.result_buffer()
        B.run_alone(t, ws, q, r, n_rows)
        assert np.array_equal(res_b[i].cpu().numpy(), r.cpu().numpy()), (i, q.template)
    assert L.device_status(0) == 0
    assert sum(1 for r in res_b if r.abs().sum().item() != 0) > n_queries // 2


@pytest.mark.gpu
@pytest.mark.parametrize("template,group_bytes", [("qb", -1), ("qb", 0), ("qb", 16384), ("qa", -1), ("mixed", 65536)])
def test_batch_group_placements_equal_alone(template, group_bytes):
    """256 queries of one form (or mixed) under shared-memory budgets that put group
    sums in shared-memory families, in L2 with per-CTA key touch bitmaps, or in L2 with
    keys written on every match: every result equals the query run alone."""
    import torch
    from mordred_b200 import _lib as L
    torch.cuda.set_device(0)
    n_rows = 2_000_003
    s = ssb.Sizes(lo_len=n_rows, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(s, 77, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    kw = {} if template == "mixed" else {"templates": (template,)}
    qs = B.generate_queries(256, seed=5, sel_lo=1e-3, sel_hi=0.3, **kw)
    res_b = [q.result_buffer() for q in qs]
    B.run_batch(t, pats, qs, res_b, n_rows, smem_group_bytes=group_bytes)
    ws = B.AloneWorkspace(s)
    for i, q in enumerate(qs):
        r = q.result_buffer()
        B.run_alone(t, ws, q, r, n_rows)
        assert np.array_equal(res_b[i].cpu().numpy(), r.cpu().numpy()), (i, q.template)
    assert L.device_status(0) == 0


@pytest.mark.gpu
def test_batch_launch_configs_and_oracle():
    import torch
    from mordred_b200 import _lib as L
    from oracle import oracle as O
    torch.cuda.set_device(0)
    n = 600_011
    s = ssb.Sizes(lo_len=n, s_len=2_000, c_len=30_000, p_len=20_000)
    t = ssb.gen_device(s, 99, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    qs = B.generate_queries(24, seed=3, sel_lo=1e-3, sel_hi=0.5)
    base = [q.result_buffer() for q in qs]
    B.run_batch(t, pats, qs, base, n)
    for threads, items in ((256, 4), (512, 4), (512, 2), (768, 1), (768, 2), (960, 1), (128, 4)):
        for stages in (2, 3):
            if True:
                res = [q.result_buffer() for q in qs]
                try:
                    B.run_batch(t, pats, qs, res, n, threads=threads, items=items, stages=stages)
                except L.MbError as e:
                    # MB_ERR_SIZE: the stage ring does not fit; MB_ERR_ARG: no such compiled variant
                    assert e.code in (1, 6)
                    continue
                for a, b in zip(res, base):
                    assert torch.equal(a, b), (threads, items, stages)
    # oracle: the same query through the CPU pipeline with filtered tables
    h = {k: v.cpu().numpy() for k, v in t.items()}
    for q, r in zip(qs, base):
        if q.template != "qb":
            continue
        hts = {}
        for name, key, val, flt, lo, hi, slots, kmin, layout in [
            ("s", "s_suppkey", None, "s_region", *q.s_region, s.s_len, 0, 0),
            ("c", "c_custkey", "c_nation", "c_region", *q.c_region, s.c_len, 0, 1),
            ("p", "p_partkey", None, "p_mfgr", *q.mfgr, s.p_len, 0, 0),
            ("d", "d_datekey", "d_year", None, 0, 0, ssb.DATE_SLOTS, ssb.DATE_MIN, 1)]:
            ht = np.zeros(2 * slots, np.int32)
            O.build_ht(h[flt] if flt else None, 1, lo, hi, h[key], h[val] if val else None, ht, slots, kmin, layout)
            hts[name] = ht
        exp = np.zeros(4 * ssb.QB_GROUPS, np.int32)
        O.star(n, filters=[dict(col=h["lo_orderdate"], mode=1, c1=q.date[0], c2=q.date[1])],
               probes=[dict(fkey=h["lo_suppkey"], ht=hts["s"], num_slots=s.s_len, layout=0),
                       dict(fkey=h["lo_custkey"], ht=hts["c"], num_slots=s.c_len, layout=1, unique_val=7, res_slot=1),
                       dict(fkey=h["lo_partkey"], ht=hts["p"], num_slots=s.p_len, layout=0),
                       dict(fkey=h["lo_orderdate"], ht=hts["d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                            layout=1, min_val=1992, unique_val=1, res_slot=0)],
               aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=ssb.QB_GROUPS, res_layout=2, res=exp)
        assert np.array_equal(r.cpu().numpy(), exp)
    assert L.device_status(0) == 0


@pytest.mark.gpu
def test_batch_wide_attributes_interval_and_table_paths():
    """Two wide attributes (orderdate over its calendar, extendedprice over a 60,000-value
    window) with 256 queries: more range end points than the interval coding takes, so
    one attribute is interval-coded and the other uses the full value table. Every
    filter-aggregate result is checked against numpy."""
    import torch
    from mordred_b200 import _lib as L
    torch.cuda.set_device(0)
    n = 2_000_003
    s = ssb.Sizes(lo_len=n, s_len=2_000, c_len=30_000, p_len=20_000)
    t = ssb.gen_device(s, 17, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    rng = np.random.default_rng(5)
    qs = B.generate_queries(256, seed=21, sel_lo=0.05, sel_hi=0.3, templates=("agg",))
    for q in qs:
        lo = 1_000_000 + int(rng.integers(0, 30_000))
        q.extra = [(B.FACT["lo_extendedprice"], lo, lo + int(rng.integers(1, 30_000)))]
    # both attributes need more end points together than the interval coding takes (768)
    def points(ranges):
        lo0, hi0 = min(r[0] for r in ranges), max(r[1] for r in ranges)
        return len({0} | {r[0] - lo0 for r in ranges if r[0] > lo0} | {r[1] + 1 - lo0 for r in ranges if r[1] < hi0})
    assert points([q.date for q in qs]) + points([q.extra[0][1:] for q in qs]) > 768
    res = [q.result_buffer() for q in qs]
    B.run_batch(t, pats, qs, res, n)
    h = {k: t[k].cpu().numpy().astype(np.int64) for k in ("lo_orderdate", "lo_discount", "lo_quantity",
                                                          "lo_extendedprice")}
    nonzero = 0
    for q, r in zip(qs, res):
        m = ((h["lo_orderdate"] >= q.date[0]) & (h["lo_orderdate"] <= q.date[1])
             & (h["lo_discount"] >= q.discount[0]) & (h["lo_discount"] <= q.discount[1])
             & (h["lo_quantity"] >= q.quantity[0]) & (h["lo_quantity"] <= q.quantity[1])
             & (h["lo_extendedprice"] >= q.extra[0][1]) & (h["lo_extendedprice"] <= q.extra[0][2]))
        exp = int((h["lo_extendedprice"][m] * h["lo_discount"][m]).sum())
        assert int(r.item()) == exp
        nonzero += exp != 0
    assert nonzero > 200
    assert L.device_status(0) == 0


@pytest.mark.gpu
def test_batch_graph_replay_and_autotune():
    """A captured batch replays to the same results as a direct run, twice; the autotuner
    picks a configuration that gives the same results too."""
    import torch
    from mordred_b200 import _lib as L
    torch.cuda.set_device(0)
    n = 3_000_017
    s = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(s, 7, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    qs = B.generate_queries(200, seed=8)
    base = [q.result_buffer() for q in qs]
    B.run_batch(t, pats, qs, base, n)
    flat, views = B.result_buffers(qs)
    plan = B.BatchPlan(t, pats, qs, views, n)
    g = plan.capture(zero=flat)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for a, b in zip(views, base):
            assert torch.equal(a.view(-1), b.view(-1))
    info = plan.autotune(reps=1)
    assert info["best"]["threads"] > 0 and len(info["timings"]) >= 2
    flat.zero_()
    plan.run()
    torch.cuda.synchronize()
    for a, b in zip(views, base):
        assert torch.equal(a.view(-1), b.view(-1))
    del g
    assert L.device_status(0) == 0


@pytest.mark.gpu
def test_batch_256_mixed_against_oracle():
    """Every query of a 256-query mixed batch (filter-aggregate, Query A, Query B forms;
    group counts 1, 175 and 7,000) against the CPU oracle running it alone with filtered
    tables — the pin for the batched kernel, not another CUDA run."""
    import torch
    from mordred_b200 import _lib as L
    from query_oracle import expected
    torch.cuda.set_device(0)
    n = 2_000_003
    s = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(s, 2027, B.BATCH_FACT, B.BATCH_DIMS)
    pats = B.build_pats(t, s)
    qs = B.generate_queries(256, seed=99, sel_lo=1e-4, sel_hi=0.3)
    flat, views = B.result_buffers(qs)
    B.BatchPlan(t, pats, qs, views, n).run()
    torch.cuda.synchronize()
    h = {k: v.cpu().numpy() for k, v in t.items()}
    nonempty = 0
    for i, q in enumerate(qs):
        exp = expected(h, s, q)
        got = views[i].cpu().numpy().reshape(-1)
        assert np.array_equal(got, exp), (i, q.template)
        nonempty += bool(np.any(exp != 0))
    assert nonempty > 200
    assert {q.template for q in qs} == {"agg", "qa", "qb"}
    assert L.device_status(0) == 0
