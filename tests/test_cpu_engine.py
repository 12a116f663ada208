"""The library's CPU operators (the CPU half of split execution) against the oracle."""
import numpy as np
import pytest

from mordred_b200 import _lib as L
from mordred_b200 import cpu, ssb
from oracle import oracle as O

FACT = ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"]
DIMS = sorted(set(ssb.QA_DIMS + ssb.QB_DIMS))


@pytest.fixture(scope="module")
def tables():
    s = ssb.Sizes(lo_len=300_007, s_len=2_000, c_len=30_000, p_len=20_000)
    return s, ssb.gen_host(s, 77, FACT, DIMS)


def _hts(s, t, builder):
    """Query B's four filtered tables built by `builder` (cpu.build_pht or the oracle)."""
    out = {}
    for name, flt, mode, c1, c2, key, val, slots, kmin, layout in [
            ("s", "s_region", L.MB_FILTER_EQ, 1, 0, "s_suppkey", None, s.s_len, 0, L.MB_HT_KEY),
            ("c", "c_region", L.MB_FILTER_EQ, 1, 0, "c_custkey", "c_nation", s.c_len, 0, L.MB_HT_KEY_VAL),
            ("p", "p_mfgr", L.MB_FILTER_EQ_OR_EQ, 0, 1, "p_partkey", None, s.p_len, 0, L.MB_HT_KEY),
            ("d", None, 0, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN, L.MB_HT_KEY_VAL)]:
        ht = np.zeros(slots if layout == L.MB_HT_KEY else 2 * slots, np.int32)
        builder(t[flt] if flt else None, mode, c1, c2, t[key], t[val] if val else None, ht, slots, kmin, layout)
        out[name] = ht
    return out


def _cpu_build(f, mode, c1, c2, key, val, ht, slots, kmin, layout):
    assert cpu.build_pht(f, mode, c1, c2, key, val, ht, slots, kmin, layout) == 0


def _orc_build(f, mode, c1, c2, key, val, ht, slots, kmin, layout):
    assert O.build_ht(f, mode, c1, c2, key, val, ht, slots, kmin, layout) == 0


def test_builds_equal_oracle(tables):
    s, t = tables
    a, b = _hts(s, t, _cpu_build), _hts(s, t, _orc_build)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # engine layout {val, row+1}
    ha, hb = np.zeros(2 * s.p_len, np.int32), np.zeros(2 * s.p_len, np.int32)
    assert cpu.build_pht(t["p_category"], L.MB_FILTER_BETWEEN, 3, 9, t["p_partkey"], t["p_brand1"], ha, s.p_len, 0,
                         L.MB_HT_VAL_OFF) == 0
    O.build_ht(t["p_category"], L.MB_FILTER_BETWEEN, 3, 9, t["p_partkey"], t["p_brand1"], hb, s.p_len, 0, 2)
    assert np.array_equal(ha, hb)


def _qb_probes(s, t, hts):
    return [dict(fkey=t["lo_suppkey"], ht=hts["s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_custkey"], ht=hts["c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
                 res_slot=1),
            dict(fkey=t["lo_partkey"], ht=hts["p"], num_slots=s.p_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_orderdate"], ht=hts["d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                 layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)]


@pytest.mark.parametrize("nthreads", [1, 0])
def test_query_b_and_filter_aggregate_equal_oracle(tables, nthreads):
    s, t = tables
    n = s.lo_len
    hts = _hts(s, t, _orc_build)
    probes = _qb_probes(s, t, hts)
    kw = dict(aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=175,
              res_layout=L.MB_RES_CRYSTAL4)
    got, exp = np.zeros(700, np.int32), np.zeros(700, np.int32)
    assert cpu.star_query(ssb.star_args(num_rows=n, probes=probes, res=got, **kw), nthreads=nthreads) == 0
    assert O.star(n, probes=probes, res=exp, **kw) == 0
    assert np.array_equal(got, exp) and got.any()
    # filter-aggregate with a count after the first two filters
    filters = [dict(col=t["lo_discount"], mode=1, c1=1, c2=3), dict(col=t["lo_quantity"], mode=1, c1=-2**31, c2=24),
               dict(col=t["lo_orderdate"], mode=1, c1=19930101, c2=19931231)]
    g1, e1 = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
    gc, ec = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
    kw = dict(filters=filters, aggr=[t["lo_extendedprice"], t["lo_discount"]], agg_op=L.MB_AGG_MUL, count_after=2)
    cpu.star_query(ssb.star_args(num_rows=n, res=g1, count=gc, **kw), nthreads=nthreads)
    O.star(n, res=e1, count=ec, **kw)
    assert g1[0] == e1[0] and gc[0] == ec[0] and g1[0] > 0


def test_engine6_dense_segments_and_offset_lists(tables):
    s, t = tables
    seg = 1 << 14
    nseg = s.lo_len // seg
    rng = np.random.default_rng(3)
    group = rng.permutation(nseg)[: nseg // 2].astype(np.int16)
    n = len(group) * seg
    hts = _hts(s, t, _orc_build)
    probes = _qb_probes(s, t, hts)
    # ENGINE6 keys in slots 1 (customer nation) and 3 (year)
    probes[1]["res_slot"], probes[3]["res_slot"] = 1, 3
    kw = dict(filters=[dict(col=t["lo_orderdate"], mode=1, c1=19940101, c2=19961231)], probes=probes,
              aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=175, res_layout=L.MB_RES_ENGINE6,
              segment_group=group, segment_size=seg)
    got, exp = np.zeros(6 * 175, np.int32), np.zeros(6 * 175, np.int32)
    cpu.star_query(ssb.star_args(num_rows=n, res=got, **kw))
    O.star(n, res=exp, **kw)
    assert np.array_equal(got, exp) and got.any()
    # an offset list: the listed rows only, against the oracle over a table of those rows
    rows = np.sort(rng.choice(n, 50_000, replace=False)).astype(np.int32)
    d_got = np.zeros(175, np.uint64)
    dk = dict(kw, res_layout=L.MB_RES_DENSE)
    cpu.star_query(ssb.star_args(num_rows=n, res=d_got, **dk), rows=rows)
    phys = (group.astype(np.int64)[rows // seg] * seg + rows % seg)
    sub = {k: np.ascontiguousarray(v[phys]) for k, v in t.items() if k.startswith("lo_")}
    sub_probes = _qb_probes(s, sub, hts)
    d_exp = np.zeros(175, np.uint64)
    O.star(len(rows), filters=[dict(col=sub["lo_orderdate"], mode=1, c1=19940101, c2=19961231)], probes=sub_probes,
           aggr=[sub["lo_revenue"], sub["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=175,
           res_layout=L.MB_RES_DENSE, res=d_exp)
    assert np.array_equal(d_got, d_exp) and d_got.any()


def test_status_and_argument_errors(tables):
    s, t = tables
    key = np.array([5, -7, 3], np.int32)  # -7 % slots is negative: reported, not written
    ht = np.zeros(16, np.int32)
    assert cpu.build_pht(None, 0, 0, 0, key, None, ht, 16, 0, L.MB_HT_KEY) == L.MB_STATUS_PROBE_RANGE
    assert ht[5] == 5 and ht[3] == 3
    res = np.zeros(1, np.uint64)
    with pytest.raises(L.MbError):
        cpu.star_query(ssb.star_args(num_rows=10, aggr=[None], res=res))
    # empty inputs are fine
    assert cpu.star_query(ssb.star_args(num_rows=0, aggr=[t["lo_revenue"]], res=res)) == 0
    assert res[0] == 0
