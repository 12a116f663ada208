"""The engine's offset-list (GPU3) kernels, the aggregate kernels and the list / min-max
builds against the oracle, and split execution in both directions: GPU select -> CPU
aggregate is in test_compact.py; here the CPU selects (mb_cpu_star_select) and the GPU
finishes the query over the list, with group values passed through from the CPU's joins."""
import ctypes as C

import numpy as np
import pytest

from mordred_b200 import _lib as L
from mordred_b200 import cpu, ssb
from oracle import oracle as O

SEG = 1 << 20


# ---- CPU: the host selection operator against the oracle's selection ---------------------

@pytest.mark.parametrize("segments", [None, [2, 0, 1]])
def test_cpu_select_matches_oracle(segments):
    rng = np.random.default_rng(11)
    nseg = 3
    n = nseg * SEG if segments is not None else 700_001
    col = rng.integers(0, 10, n).astype(np.int32)
    key = rng.integers(1, 5000, n).astype(np.int32)
    key2 = rng.integers(1, 300, n).astype(np.int32)
    dk = np.arange(1, 5001, dtype=np.int32)
    ht = np.zeros(2 * 5000, np.int32)
    O.build_ht((dk % 3).astype(np.int32), 1, 1, 2, dk, (dk % 7).astype(np.int32), ht, 5000, 0, 2)
    ht2 = np.zeros(2 * 300, np.int32)
    d2 = np.arange(1, 301, dtype=np.int32)
    O.build_ht((d2 % 2).astype(np.int32), 0, 1, 0, d2, (d2 * 3).astype(np.int32), ht2, 300, 0, 1)
    seg = np.array(segments, np.int16) if segments is not None else None
    kw = dict(filters=[dict(col=col, mode=1, c1=2, c2=8)],
              probes=[dict(fkey=key, ht=ht, num_slots=5000, layout=2), dict(fkey=key2, ht=ht2, num_slots=300, layout=1)])
    extra = dict(segment_group=seg, segment_size=SEG) if seg is not None else {}
    a = ssb.star_args(num_rows=n, aggr=[col], res_layout=0, res=np.zeros(1, np.int64), **kw, **extra)
    lo, dims, st = cpu.star_select(a)
    olo, odims, k, ost = O.select(n, **kw, **extra)
    assert st == 0 and ost == 0 and len(lo) == k
    assert np.array_equal(lo, olo)
    for d, od in zip(dims, odims):
        assert np.array_equal(d, od)
    # capacity: counted, not written
    lo2, _, st2 = cpu.star_select(a, capacity=10)
    assert len(lo2) == 10 and st2 & L.MB_STATUS_OVERFLOW and np.array_equal(lo2, olo[:10])


def test_oracle_list_form_equals_whole_query():
    """The oracle's offset-list form with passed-through group values gives the whole query's
    answer: select with the supplier probe, then aggregate the list grouping by the
    supplier's nation read at the passed dimension row."""
    rng = np.random.default_rng(3)
    n = 200_003
    s_len = 3000
    lo_supp = rng.integers(1, s_len + 1, n).astype(np.int32)
    rev = rng.integers(90_100, 10_494_950, n).astype(np.int32)
    od = rng.integers(0, 100, n).astype(np.int32)
    sk = np.arange(1, s_len + 1, dtype=np.int32)
    nation = rng.integers(0, 25, s_len).astype(np.int32)
    region = (nation // 5).astype(np.int32)
    ht = np.zeros(2 * s_len, np.int32)
    O.build_ht(region, 1, 1, 3, sk, nation, ht, s_len, 0, 2)
    whole = np.zeros(6 * 25, np.int32)
    O.star(n, filters=[dict(col=od, mode=1, c1=10, c2=60)],
           probes=[dict(fkey=lo_supp, ht=ht, num_slots=s_len, layout=2, unique_val=1, res_slot=0)],
           aggr=[rev], agg_op=0, total_val=25, res_layout=1, res=whole)
    lo, dims, k, _ = O.select(n, filters=[dict(col=od, mode=1, c1=10, c2=60)],
                              probes=[dict(fkey=lo_supp, ht=ht, num_slots=s_len, layout=2)])
    part = np.zeros(6 * 25, np.int32)
    O.star(k, rows=lo, probes=[dict(fkey=dims[0], ht=nation, num_slots=s_len, layout=O.LAYOUT_PASS, unique_val=1,
                                    res_slot=0)],
           aggr=[rev], agg_op=0, total_val=25, res_layout=1, res=part)
    assert np.array_equal(whole, part)


# ---- GPU ---------------------------------------------------------------------------------------

def _cache_setup(seed=21, nseg=3, tail=54_321):
    """Fact columns and the dimension columns in a shuffled segment cache (slot arrays per
    column), engine hash tables on the GPU and the host."""
    import torch
    lo_len = (nseg - 1) * SEG + tail
    s = ssb.Sizes(lo_len=lo_len, s_len=8_000, c_len=90_000, p_len=150_000)
    fact = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost", "lo_quantity",
            "lo_discount", "lo_extendedprice"]
    dims = ssb.QB_DIMS + ["s_nation", "p_brand1", "p_category"]
    t = ssb.gen_device(s, seed, fact, dims)
    h = {k: v.cpu().numpy() for k, v in t.items()}
    cols = [(name, lo_len) for name in fact] + [(name, len(h[name])) for name in dims]
    nslots = sum((n + SEG - 1) // SEG for _, n in cols) + 2
    rng = np.random.default_rng(seed)
    perm = list(rng.permutation(nslots))
    cache = torch.zeros(nslots * SEG, dtype=torch.int32, device="cuda")
    col_idx = {}
    for name, n in cols:
        sl = []
        for sg in range((n + SEG - 1) // SEG):
            slot = int(perm.pop())
            lo, hi = sg * SEG, min((sg + 1) * SEG, n)
            cache[slot * SEG: slot * SEG + (hi - lo)] = t[name][lo:hi]
            sl.append(slot)
        col_idx[name] = torch.tensor(sl, dtype=torch.int32, device="cuda")
    hts = {}
    specs = [("s", "s_suppkey", "s_nation", "s_region", 1, 0, 2, s.s_len, 0),
             ("c", "c_custkey", "c_nation", "c_region", 1, 1, 3, s.c_len, 0),
             ("p", "p_partkey", "p_brand1", "p_mfgr", 2, 0, 1, s.p_len, 0),
             ("d", "d_datekey", "d_year", None, 0, 0, 0, ssb.DATE_SLOTS, 19920101)]
    for name, key, val, flt, mode, c1, c2, slots, kmin in specs:
        ref = np.zeros(2 * slots, np.int32)
        O.build_ht(h[flt] if flt else None, mode, c1, c2, h[key], h[val], ref, slots, kmin, 2)
        hts[name] = (torch.from_numpy(ref).cuda(), ref, slots, kmin)
    return s, t, h, cache, col_idx, hts, lo_len


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).cuda()


@pytest.mark.gpu
def test_split_cpu_select_gpu_group_by_with_passed_groups():
    """CPU-select -> GPU-aggregate: the CPU filters orderdate and joins supplier and part
    (recording the dimension rows they matched); the GPU runs filter_probe_group_by_GPU3 over
    the list, filtering quantity, probing customer and date, and grouping by the supplier's
    nation read at the passed dimension row, the customer's nation and the year. Equal to the
    oracle's whole query, and to the oracle's own list form."""
    import torch
    s, t, h, cache, ci, hts, n = _cache_setup()
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    # CPU half: filter + supplier and part probes -> offset list with dimension rows
    a = ssb.star_args(num_rows=n, filters=[dict(col=h["lo_orderdate"], mode=1, c1=19930301, c2=19960131)],
                      probes=[dict(fkey=h["lo_suppkey"], ht=hts["s"][1], num_slots=s.s_len, layout=2),
                              dict(fkey=h["lo_partkey"], ht=hts["p"][1], num_slots=s.p_len, layout=2)],
                      aggr=[h["lo_revenue"]], res_layout=0, res=np.zeros(1, np.int64))
    lo, (d_s, d_p), st = cpu.star_select(a)
    assert st == 0 and len(lo) > 1000
    lo_d, ds_d, dp_d = _dev(lo), _dev(d_s), _dev(d_p)
    off = L.MbOffsetGPU(lo_d.data_ptr(), ds_d.data_ptr(), None, dp_d.data_ptr(), None)
    f = L.MbFilterArgsGPU(None, ci["lo_quantity"].data_ptr(), 0, 0, 3, 44, 1, 1)
    p = L.MbProbeArgsGPU(None, ci["lo_custkey"].data_ptr(), None, ci["lo_orderdate"].data_ptr(),
                         None, hts["c"][0].data_ptr(), None, hts["d"][0].data_ptr(),
                         0, s.c_len, 0, ssb.DATE_SLOTS, 0, 0, 0, 19920101)
    # group (s_nation passed through, c_nation, -, year): s*175 + c*7 + (year - 1992), one
    # key tuple per group; the part slot was joined on the CPU and is not grouped
    total = 25 * 175
    g = L.MbGroupbyArgsGPU(ci["lo_revenue"].data_ptr(), ci["lo_supplycost"].data_ptr(),
                           ci["s_nation"].data_ptr(), None, None, None,
                           0, 0, 0, 1992, 175, 7, 0, 1, total, 0)
    res = torch.zeros(6 * total, dtype=torch.int32, device="cuda")
    L.call("mb_filter_probe_group_by_GPU3", cache.data_ptr(), C.byref(off), C.byref(f), C.byref(p), C.byref(g),
           len(lo), res.data_ptr(), ssb._stream())
    # oracle: the whole query in one pass
    exp = np.zeros(6 * total, np.int32)
    ost = O.star(n, filters=[dict(col=h["lo_orderdate"], mode=1, c1=19930301, c2=19960131),
                             dict(col=h["lo_quantity"], mode=1, c1=3, c2=44)],
                 probes=[dict(fkey=h["lo_suppkey"], ht=hts["s"][1], num_slots=s.s_len, layout=2, unique_val=175,
                              res_slot=0),
                         dict(fkey=h["lo_custkey"], ht=hts["c"][1], num_slots=s.c_len, layout=2, unique_val=7,
                              res_slot=1),
                         dict(fkey=h["lo_partkey"], ht=hts["p"][1], num_slots=s.p_len, layout=2),
                         dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=ssb.DATE_SLOTS, key_min=19920101,
                              layout=2, min_val=1992, unique_val=1, res_slot=3)],
                 aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=total, res_layout=1, res=exp)
    assert ost == 0
    assert L.device_status(0, clear=True) == 0
    assert np.array_equal(res.cpu().numpy(), exp)
    assert (exp.reshape(-1, 6)[:, 4:6] != 0).any()
    # and the oracle's own list form agrees
    exp2 = np.zeros(6 * total, np.int32)
    O.star(len(lo), rows=lo, filters=[dict(col=h["lo_quantity"], mode=1, c1=3, c2=44)],
           probes=[dict(fkey=d_s, ht=h["s_nation"], num_slots=s.s_len, layout=O.LAYOUT_PASS, unique_val=175,
                        res_slot=0),
                   dict(fkey=h["lo_custkey"], ht=hts["c"][1], num_slots=s.c_len, layout=2, unique_val=7, res_slot=1),
                   dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=ssb.DATE_SLOTS, key_min=19920101, layout=2,
                        min_val=1992, unique_val=1, res_slot=3)],
           aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=total, res_layout=1, res=exp2)
    assert np.array_equal(exp, exp2)


@pytest.mark.gpu
def test_list_forms_probe_group_by_group_by_and_aggregates():
    import torch
    s, t, h, cache, ci, hts, n = _cache_setup(seed=8, nseg=2, tail=99_999)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    st = ssb._stream()
    # an offset list from the GPU's own selection (mb_filter_probe_GPU2: date filter, supplier join)
    lo_d = torch.zeros(n, dtype=torch.int32, device="cuda")
    ds_d = torch.zeros(n, dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    f = L.MbFilterArgsGPU(ci["lo_orderdate"].data_ptr(), None, 19940101, 19951231, 0, 0, 1, 0)
    ps = L.MbProbeArgsGPU(ci["lo_suppkey"].data_ptr(), None, None, None, hts["s"][0].data_ptr(), None, None, None,
                          s.s_len, 0, 0, 0, 0, 0, 0, 0)
    out = L.MbOffsetGPU(lo_d.data_ptr(), ds_d.data_ptr(), None, None, None)
    L.call("mb_filter_probe_GPU2", cache.data_ptr(), C.byref(f), C.byref(ps), C.byref(out), n, total.data_ptr(), 0,
           None, st)
    k = int(total.item())
    assert k > 1000
    lo = lo_d[:k].cpu().numpy()
    d_s = ds_d[:k].cpu().numpy()
    off = L.MbOffsetGPU(lo_d.data_ptr(), ds_d.data_ptr(), None, None, None)
    # probe_group_by_GPU3: date probe, group (s_nation passed through, year)
    p = L.MbProbeArgsGPU(None, None, None, ci["lo_orderdate"].data_ptr(), None, None, None, hts["d"][0].data_ptr(),
                         0, 0, 0, ssb.DATE_SLOTS, 0, 0, 0, 19920101)
    g = L.MbGroupbyArgsGPU(ci["lo_revenue"].data_ptr(), None, ci["s_nation"].data_ptr(), None, None, None,
                           0, 0, 0, 1992, 7, 0, 0, 1, 175, 0)
    res = torch.zeros(6 * 175, dtype=torch.int32, device="cuda")
    L.call("mb_probe_group_by_GPU3", cache.data_ptr(), C.byref(off), C.byref(p), C.byref(g), k, res.data_ptr(), st)
    exp = np.zeros(6 * 175, np.int32)
    O.star(k, rows=lo, probes=[dict(fkey=d_s, ht=h["s_nation"], num_slots=s.s_len, layout=O.LAYOUT_PASS,
                                    unique_val=7, res_slot=0),
                               dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=ssb.DATE_SLOTS,
                                    key_min=19920101, layout=2, min_val=1992, unique_val=1, res_slot=3)],
           aggr=[h["lo_revenue"]], agg_op=0, total_val=175, res_layout=1, res=exp)
    assert np.array_equal(res.cpu().numpy(), exp)
    # groupByGPU: group by the passed nation only, SUM(revenue - supplycost)
    g2 = L.MbGroupbyArgsGPU(ci["lo_revenue"].data_ptr(), ci["lo_supplycost"].data_ptr(), ci["s_nation"].data_ptr(),
                            None, None, None, 0, 0, 0, 0, 1, 0, 0, 0, 25, 0)
    res2 = torch.zeros(6 * 25, dtype=torch.int32, device="cuda")
    L.call("mb_groupByGPU", cache.data_ptr(), C.byref(off), C.byref(g2), k, res2.data_ptr(), st)
    exp2 = np.zeros(6 * 25, np.int32)
    O.star(k, rows=lo, probes=[dict(fkey=d_s, ht=h["s_nation"], num_slots=s.s_len, layout=O.LAYOUT_PASS,
                                    unique_val=1, res_slot=0)],
           aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=25, res_layout=1, res=exp2)
    assert np.array_equal(res2.cpu().numpy(), exp2)
    # aggregationGPU: SUM(extendedprice * discount) over the list at res[4]
    g3 = L.MbGroupbyArgsGPU(ci["lo_extendedprice"].data_ptr(), ci["lo_discount"].data_ptr(), None, None, None, None,
                            0, 0, 0, 0, 0, 0, 0, 0, 1, 1)
    res3 = torch.zeros(6, dtype=torch.int32, device="cuda")
    L.call("mb_aggregationGPU", cache.data_ptr(), lo_d.data_ptr(), C.byref(g3), k, res3.data_ptr(), st)
    exp3 = np.zeros(1, np.uint64)
    O.star(k, rows=lo, aggr=[h["lo_extendedprice"], h["lo_discount"]], agg_op=2, res_layout=0, res=exp3)
    assert int(res3.cpu().numpy()[4:6].view(np.uint64)[0]) == int(exp3[0])
    # probe_aggr_GPU3 (date probe) and filter_probe_aggr_GPU3 (the second filter only)
    for fn, fa in (("mb_probe_aggr_GPU3", None),
                   ("mb_filter_probe_aggr_GPU3", L.MbFilterArgsGPU(ci["lo_discount"].data_ptr(),
                                                                   ci["lo_quantity"].data_ptr(), 0, 0, 10, 30, 1, 1))):
        r = torch.zeros(6, dtype=torch.int32, device="cuda")
        args = [cache.data_ptr(), C.byref(off)] + ([C.byref(fa)] if fa is not None else []) + \
               [C.byref(p), C.byref(g3), k, r.data_ptr(), st]
        L.call(fn, *args)
        e = np.zeros(1, np.uint64)
        filters = [dict(col=h["lo_quantity"], mode=1, c1=10, c2=30)] if fa is not None else []
        O.star(k, rows=lo, filters=filters,
               probes=[dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=ssb.DATE_SLOTS, key_min=19920101,
                            layout=2)],
               aggr=[h["lo_extendedprice"], h["lo_discount"]], agg_op=2, res_layout=0, res=e)
        assert int(r.cpu().numpy()[4:6].view(np.uint64)[0]) == int(e[0]), fn
    # probe_aggr_GPU2 over the whole segment range
    r = torch.zeros(6, dtype=torch.int32, device="cuda")
    L.call("mb_probe_aggr_GPU2", cache.data_ptr(), C.byref(p), C.byref(g3), n, r.data_ptr(), 0, None, st)
    e = np.zeros(1, np.uint64)
    O.star(n, probes=[dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=ssb.DATE_SLOTS, key_min=19920101,
                           layout=2)],
           aggr=[h["lo_extendedprice"], h["lo_discount"]], agg_op=2, res_layout=0, res=e)
    assert int(r.cpu().numpy()[4:6].view(np.uint64)[0]) == int(e[0])
    assert L.device_status(0, clear=True) == 0


@pytest.mark.gpu
def test_star_query_rows_generic_direct_columns():
    """mb_star_query with an offset list over plain device columns, every result layout."""
    import torch
    rng = np.random.default_rng(5)
    n = 1_500_007
    s = ssb.Sizes(lo_len=n, s_len=5_000, c_len=60_000, p_len=90_000)
    t = ssb.gen_device(s, 4, ssb.QB_FACT, ssb.QB_DIMS)
    h = {k: v.cpu().numpy() for k, v in t.items()}
    rows = np.sort(rng.choice(n, 400_000, replace=False)).astype(np.int32)
    rng.shuffle(rows)
    ht_c = np.zeros(2 * s.c_len, np.int32)
    O.build_ht(h["c_region"], 1, 1, 3, h["c_custkey"], h["c_nation"], ht_c, s.c_len, 0, 1)
    ht_d = np.zeros(2 * ssb.DATE_SLOTS, np.int32)
    O.build_ht(None, 0, 0, 0, h["d_datekey"], h["d_year"], ht_d, ssb.DATE_SLOTS, ssb.DATE_MIN, 1)
    rows_d, htc_d, htd_d = _dev(rows), _dev(ht_c), _dev(ht_d)
    for layout, total in ((L.MB_RES_CRYSTAL4, 175), (L.MB_RES_DENSE, 175), (L.MB_RES_SCALAR, 1)):
        res = torch.zeros(4 * 175 if layout == L.MB_RES_CRYSTAL4 else 2 * 175, dtype=torch.int32, device="cuda")
        probes = [dict(fkey=t["lo_custkey"], ht=htc_d, num_slots=s.c_len, layout=1, unique_val=7, res_slot=1),
                  dict(fkey=t["lo_orderdate"], ht=htd_d, num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN, layout=1,
                       min_val=1992, unique_val=1, res_slot=0)]
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        a = ssb.star_args(num_rows=len(rows), filters=[dict(col=t["lo_revenue"], mode=1, c1=200_000, c2=9_000_000)],
                          probes=probes, aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB,
                          total_val=total, res_layout=layout, res=res, count=cnt, count_after=1, rows=rows_d)
        ssb.star_query(a)
        exp = np.zeros(res.numel(), np.int32)
        ecnt = np.zeros(1, np.uint64)
        O.star(len(rows), rows=rows, filters=[dict(col=h["lo_revenue"], mode=1, c1=200_000, c2=9_000_000)],
               probes=[dict(fkey=h["lo_custkey"], ht=ht_c, num_slots=s.c_len, layout=1, unique_val=7, res_slot=1),
                       dict(fkey=h["lo_orderdate"], ht=ht_d, num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                            layout=1, min_val=1992, unique_val=1, res_slot=0)],
               aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=total, res_layout=layout, res=exp,
               count=ecnt, count_after=1)
        assert np.array_equal(res.cpu().numpy(), exp), layout
        assert int(cnt.item()) == int(ecnt[0])
    assert L.device_status(0, clear=True) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("k", [0, 1, 31, 33, 100_003])
def test_star_query_rows_edge_sizes_and_large_group_array(k):
    """Offset lists of 0, 1 and around one warp of entries, and a list form whose group
    array (12,000 groups, engine layout) is too large for shared memory, against the
    oracle."""
    import torch
    rng = np.random.default_rng(k + 1)
    n = 300_007
    key = rng.integers(1, 50_001, n).astype(np.int32)
    val = rng.integers(-1000, 1_000_000, n).astype(np.int32)
    dk = np.arange(1, 50_001, dtype=np.int32)
    ht = np.zeros(2 * 50_000, np.int32)
    O.build_ht((dk % 4).astype(np.int32), 1, 0, 2, dk, (dk * 7 % 12_000).astype(np.int32), ht, 50_000, 0, 1)
    rows = rng.choice(n, k, replace=False).astype(np.int32)
    res = torch.zeros(6 * 12_000, dtype=torch.int32, device="cuda")
    probes = lambda kk, hh: [dict(fkey=kk, ht=hh, num_slots=50_000, layout=1, unique_val=1, res_slot=2)]
    a = ssb.star_args(num_rows=k, probes=probes(_dev(key), _dev(ht)), aggr=[_dev(val)], agg_op=L.MB_AGG_SUM,
                      total_val=12_000, res_layout=L.MB_RES_ENGINE6, res=res, rows=_dev(rows))
    ssb.star_query(a)
    exp = np.zeros(6 * 12_000, np.int32)
    O.star(k, rows=rows, probes=probes(key, ht), aggr=[val], agg_op=0, total_val=12_000, res_layout=1, res=exp)
    assert np.array_equal(res.cpu().numpy(), exp)
    assert exp.any() if k >= 31 else True
    assert L.device_status(0, clear=True) == 0


@pytest.mark.gpu
def test_list_builds_and_minmax():
    """build_GPU3 and build_GPU_minmax2 over a list of dimension rows, build_GPU_minmax over a
    segment range, against the oracle (tables and key ranges)."""
    import torch
    s, t, h, cache, ci, hts, n = _cache_setup(seed=13, nseg=1, tail=1000)
    L.call("mb_init", 0)
    st = ssb._stream()
    rng = np.random.default_rng(2)
    dim_rows = np.sort(rng.choice(s.p_len, 20_000, replace=False)).astype(np.int32)
    rng.shuffle(dim_rows)
    dr = _dev(dim_rows)
    b = L.MbBuildArgsGPU(ci["p_partkey"].data_ptr(), ci["p_brand1"].data_ptr(), s.p_len, 0, s.p_len)
    ht = torch.zeros(2 * s.p_len, dtype=torch.int32, device="cuda")
    L.call("mb_build_GPU3", cache.data_ptr(), dr.data_ptr(), None, C.byref(b), len(dim_rows), ht.data_ptr(), st)
    ref = np.zeros(2 * s.p_len, np.int32)
    O.build_rows(None, 0, 0, 0, h["p_partkey"], h["p_brand1"], dim_rows, len(dim_rows), ref, s.p_len, 0)
    assert np.array_equal(ht.cpu().numpy(), ref)
    # minmax2 (list) and minmax (segment range, filtered), each into fresh (INT_MAX, INT_MIN) words
    for form in ("minmax2", "minmax"):
        ht = torch.zeros(2 * s.p_len, dtype=torch.int32, device="cuda")
        mm = torch.tensor([2**31 - 1, -2**31], dtype=torch.int32, device="cuda")
        ref = np.zeros(2 * s.p_len, np.int32)
        emm = np.array([2**31 - 1, -2**31], np.int32)
        if form == "minmax2":
            L.call("mb_build_GPU_minmax2", cache.data_ptr(), dr.data_ptr(), None, C.byref(b), len(dim_rows),
                   ht.data_ptr(), mm.data_ptr(), mm[1:].data_ptr(), st)
            O.build_rows(None, 0, 0, 0, h["p_partkey"], h["p_brand1"], dim_rows, len(dim_rows), ref, s.p_len, 0,
                         minmax=emm, val_min=0, val_max=s.p_len)
        else:
            f = L.MbFilterArgsGPU(ci["p_category"].data_ptr(), None, 4, 11, 0, 0, 1, 0)
            L.call("mb_build_GPU_minmax", cache.data_ptr(), C.byref(f), C.byref(b), s.p_len, ht.data_ptr(),
                   mm.data_ptr(), mm[1:].data_ptr(), 0, None, st)
            O.build_rows(h["p_category"], 1, 4, 11, h["p_partkey"], h["p_brand1"], None, s.p_len, ref, s.p_len, 0,
                         minmax=emm, val_min=0, val_max=s.p_len)
        assert np.array_equal(ht.cpu().numpy(), ref), form
        assert mm.cpu().numpy().tolist() == emm.tolist(), form
    assert L.device_status(0, clear=True) == 0
