"""CPU tests: the oracle against the reference's own answers and hand-computed cases."""
import datetime as dt
import json
import os

import numpy as np
import pytest

from mordred_b200 import ssb
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_ssb.json")))
ALL_FACT = ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"]
ALL_DIMS = ssb.QB_DIMS + ["p_brand1", "p_category"]


def gen(case):
    s = ssb.Sizes(lo_len=case["lo_len"], s_len=case["s_len"], c_len=case["c_len"], p_len=case["p_len"],
                  d_len=case["d_len"])
    return ssb.gen_host(s, case["seed"], ALL_FACT, ALL_DIMS)


@pytest.mark.parametrize("case", GOLD["cases"], ids=lambda c: f"seed{c['seed']}_n{c['lo_len']}")
def test_oracle_matches_reference_golden(case):
    t = gen(case)
    assert O.q11(t) == case["q11_revenue"]
    res, st = O.q21(t, case["d_val_len"])
    assert st == 0
    assert O.q21_groups(res) == [tuple(g) for g in case["q21_groups"]]
    res4, st = O.q41(t, case["d_val_len"])
    assert st == 0
    assert ssb.crystal4_groups(res4) == [tuple(g) for g in case["q41_groups"]]


@pytest.mark.skipif(not O.ref_available(21), reason="reference CPU engine not built here")
def test_oracle_matches_reference_binaries_fresh_seed():
    case = dict(seed=12345, lo_len=300_001, s_len=3_000, c_len=45_000, p_len=50_000, d_len=2556)
    t = gen(case)
    d_val_len = ssb.REFERENCE_DATE_SLOTS
    lines, _ = O.run_ref(11, **case, threads=4)
    assert O.parse_ref_revenue(lines)[-1] == O.q11(t)
    lines, _ = O.run_ref(21, **case, threads=4)
    assert O.parse_ref_groups(lines) == O.q21_groups(O.q21(t, d_val_len)[0])
    lines, _ = O.run_ref(41, **case, threads=4)
    assert O.parse_ref_groups(lines) == ssb.crystal4_groups(O.q41(t, d_val_len)[0])


def test_q11_known_answer():
    # q11.cpp:37-46: 19930000 < orderdate < 19940000, 1 <= discount <= 3, quantity < 25
    od = np.array([19930101, 19931231, 19930000, 19940000, 19930615, 19930615, 19930701, 19930702], np.int32)
    disc = np.array([1, 3, 2, 2, 0, 4, 3, 2], np.int32)
    qty = np.array([24, 1, 10, 10, 10, 10, 24, 25], np.int32)
    price = np.array([100, 10494950, 5, 5, 7, 7, 1_000_000_000, 9], np.int32)
    t = {"lo_orderdate": od, "lo_discount": disc, "lo_quantity": qty, "lo_extendedprice": price}
    # the 1e9 * 3 product is formed in int32 (wraps negative) and then widened
    wrapped = (1_000_000_000 * 3 + 2**31) % 2**32 - 2**31
    expect = (100 * 1 + 10494950 * 3 + wrapped) % 2**64
    assert O.q11(t) == expect


def _tiny_q21_tables(d_rows):
    return {
        "s_suppkey": np.array([1, 2, 3, 4], np.int32), "s_region": np.array([1, 0, 1, 1], np.int32),
        "p_partkey": np.array([1, 2, 3], np.int32), "p_category": np.array([1, 1, 0], np.int32),
        "p_brand1": np.array([5, 0, 9], np.int32),
        "d_datekey": np.array([r[0] for r in d_rows], np.int32), "d_year": np.array([r[1] for r in d_rows], np.int32),
        "lo_suppkey": np.array([1, 2, 4, 3, 4, 4], np.int32),
        "lo_partkey": np.array([1, 1, 3, 2, 1, 1], np.int32),
        "lo_orderdate": np.array([19920101, 19920101, 19950615, 19981231, 19950615, 19950615], np.int32),
        "lo_revenue": np.array([10, 11, 12, 7, 2**31 - 1, 2**31 - 1], np.int32),
    }


def test_q21_known_answer_and_date_wrap():
    dates = [(19920101, 1992), (19950615, 1995), (19981231, 1998)]
    t = _tiny_q21_tables(dates)
    # supplier 4 hashes to slot 0 (4 % 4); part 3 (category 0) is not built; brand 0 is a valid payload
    res, st = O.q21(t, ssb.DATE_SLOTS)
    assert st == 0
    assert O.q21_groups(res) == [(1992, 5, 10), (1995, 5, 2 * (2**31 - 1)), (1998, 0, 7)]
    # with the reference's 61,130 date slots 19981231 lands on 19920101's slot and,
    # built last, relabels the 1992 row as 1998 (the hazard the 61,131-slot table removes)
    res, st = O.q21(t, ssb.REFERENCE_DATE_SLOTS)
    assert O.q21_groups(res) == [(1995, 5, 2 * (2**31 - 1)), (1998, 0, 7), (1998, 5, 10)]


def test_q41_known_answer_signed():
    t = {
        "s_suppkey": np.array([1, 2], np.int32), "s_region": np.array([1, 1], np.int32),
        "c_custkey": np.array([1, 2, 3], np.int32), "c_region": np.array([1, 1, 0], np.int32),
        "c_nation": np.array([5, 9, 2], np.int32),
        "p_partkey": np.array([1, 2, 3], np.int32), "p_mfgr": np.array([0, 1, 2], np.int32),
        "d_datekey": np.array([19920101, 19970301], np.int32), "d_year": np.array([1992, 1997], np.int32),
        "lo_suppkey": np.array([1, 2, 2, 1, 1], np.int32),
        "lo_custkey": np.array([1, 2, 3, 2, 1], np.int32),
        "lo_partkey": np.array([1, 2, 1, 3, 2], np.int32),
        "lo_orderdate": np.array([19920101, 19970301, 19970301, 19970301, 19920101], np.int32),
        "lo_revenue": np.array([100, 54_000, 1, 1, 200], np.int32),
        "lo_supplycost": np.array([600_000, 1, 1, 1, 50], np.int32),
    }
    res, st = O.q41(t, ssb.DATE_SLOTS)
    assert st == 0
    # rows 0 and 4 share (1992, nation 5): (100 - 600000) + (200 - 50)
    assert ssb.crystal4_groups(res) == [(1992, 5, 100 - 600_000 + 150), (1997, 9, 54_000 - 1)]


def test_empty_inputs():
    case = dict(seed=3, lo_len=0, s_len=10, c_len=10, p_len=10, d_len=2557)
    s = ssb.Sizes(lo_len=0, s_len=10, c_len=10, p_len=10)
    t = ssb.gen_host(s, 3, ALL_FACT, ALL_DIMS)
    assert O.q11(t) == 0
    assert O.q21_groups(O.q21(t, ssb.DATE_SLOTS)[0]) == []
    assert ssb.crystal4_groups(O.q41(t, ssb.DATE_SLOTS)[0]) == []


def _crystal_tables(t, d_slots, category=1, region=1, layout_p=1):
    s_ht = np.zeros(len(t["s_suppkey"]), np.int32)
    O.build_ht(t["s_region"], 0, region, 0, t["s_suppkey"], None, s_ht, len(s_ht), 0, 0)
    p_ht = np.zeros(2 * len(t["p_partkey"]), np.int32)
    O.build_ht(t["p_category"], 0, category, 0, t["p_partkey"], t["p_brand1"], p_ht, len(t["p_partkey"]), 0, 1)
    d_ht = np.zeros(2 * d_slots, np.int32)
    O.build_ht(None, 0, 0, 0, t["d_datekey"], t["d_year"], d_ht, d_slots, 19920101, 1)
    return s_ht, p_ht, d_ht


def test_generic_pipeline_equals_q21_restatement():
    case = dict(seed=9, lo_len=50_000, s_len=500, c_len=900, p_len=4_000, d_len=2557)
    t = gen(case)
    s_ht, p_ht, d_ht = _crystal_tables(t, ssb.DATE_SLOTS)
    res = np.zeros(4 * ssb.QA_GROUPS, np.int32)
    st = O.star(case["lo_len"], probes=[
        dict(fkey=t["lo_suppkey"], ht=s_ht, num_slots=case["s_len"], layout=0),
        dict(fkey=t["lo_partkey"], ht=p_ht, num_slots=case["p_len"], layout=1, unique_val=7, res_slot=1),
        dict(fkey=t["lo_orderdate"], ht=d_ht, num_slots=ssb.DATE_SLOTS, key_min=19920101, layout=1,
             min_val=1992, unique_val=1, res_slot=0)],
        aggr=[t["lo_revenue"]], agg_op=0, total_val=ssb.QA_GROUPS, res_layout=2, res=res)
    assert st == 0
    assert ssb.crystal4_groups(res) == O.q21_groups(O.q21(t, ssb.DATE_SLOTS)[0])


def test_engine_layout_pipeline_equals_q41_restatement():
    case = dict(seed=11, lo_len=60_000, s_len=700, c_len=3_000, p_len=2_000, d_len=2557)
    t = gen(case)
    n = case["lo_len"]
    # engine layout {val, row+1}; slot order 1..4 = supplier, customer, part, date
    hts = {}
    for name, key, val, flt, mode, c1, c2, slots, kmin in [
        ("s", "s_suppkey", None, "s_region", 1, 1, 1, case["s_len"], 0),
        ("c", "c_custkey", "c_nation", "c_region", 1, 1, 1, case["c_len"], 0),
        ("p", "p_partkey", None, "p_mfgr", 2, 0, 1, case["p_len"], 0),
        ("d", "d_datekey", "d_year", None, 0, 0, 0, ssb.DATE_SLOTS, 19920101),
    ]:
        ht = np.zeros(2 * slots, np.int32)
        O.build_ht(t[flt] if flt else None, mode, c1, c2, t[key], t[val] if val else None, ht, slots, kmin, 2)
        hts[name] = (ht, slots, kmin)
    res = np.zeros(6 * ssb.QB_GROUPS, np.int32)
    probes = []
    for slot, (name, fk, mn, uq) in enumerate([("s", "lo_suppkey", 0, 0), ("c", "lo_custkey", 0, 7),
                                                 ("p", "lo_partkey", 0, 0), ("d", "lo_orderdate", 1992, 1)]):
        ht, slots, kmin = hts[name]
        probes.append(dict(fkey=t[fk], ht=ht, num_slots=slots, key_min=kmin, layout=2, min_val=mn, unique_val=uq,
                           res_slot=slot))
    st = O.star(n, probes=probes, aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=1, total_val=ssb.QB_GROUPS,
                res_layout=1, res=res)
    assert st == 0
    # engine res keeps (g1..g4) = (supplier val 0, nation, part val 0, year)
    eng = [(g[3], g[1], g[4]) for g in ssb.engine6_groups(res)]
    assert sorted(eng) == ssb.crystal4_groups(O.q41(t, ssb.DATE_SLOTS)[0])


def _py_star(n, filters, probes, aggr, agg_op, total, res_layout):
    """Straight Python loop of the generic pipeline (small inputs only)."""
    def i32(x):
        return (x + 2**31) % 2**32 - 2**31
    groups, scalar = {}, 0
    for r in range(n):
        ok = True
        for f in filters:
            x = int(f["col"][r])
            m = f.get("mode", 1)
            ok = (f["c1"] <= x <= f["c2"]) if m == 1 else (x == f["c1"]) if m == 0 else (x in (f["c1"], f["c2"]))
            if not ok:
                break
        if not ok:
            continue
        gv = []
        for q in probes:
            d = int(q["fkey"][r]) - q.get("key_min", 0)
            h = int(np.fmod(d, q["num_slots"]))
            if h < 0:
                ok = False
                break
            if q["layout"] == 0:
                ok = int(q["ht"][h]) != 0
                gv.append(0)
            else:
                lo, hi = int(q["ht"][2 * h]), int(q["ht"][2 * h + 1])
                ok = lo != 0 or hi != 0
                gv.append(hi if q["layout"] == 1 else lo)
            if not ok:
                break
        if not ok:
            continue
        a0 = int(aggr[0][r])
        v = a0 if agg_op == 0 else i32(a0 - int(aggr[1][r])) if agg_op == 1 else i32(a0 * int(aggr[1][r]))
        if res_layout == 0:
            scalar += v
            continue
        hh = i32(sum(i32(g - q.get("min_val", 0)) * q.get("unique_val", 0) for g, q in zip(gv, probes)))
        g = int(np.fmod(hh, total))
        groups[g] = groups.get(g, 0) + v
    return scalar % 2**64, {g: (s + 2**63) % 2**64 - 2**63 for g, s in groups.items()}


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_generic_pipeline_against_python_loop(seed):
    rng = np.random.default_rng(seed)
    n, slots = 3000, 97
    col = lambda lo, hi: rng.integers(lo, hi + 1, n).astype(np.int32)
    f0, f1 = col(0, 20), col(-5, 5)
    k0, k1 = col(-3, 2 * slots), col(1, slots)
    a0, a1 = col(-(2**31), 2**31 - 1), col(-1000, 1000)
    ht0 = np.zeros(slots, np.int32)
    ht0[rng.integers(0, slots, 40)] = 1
    ht1 = np.zeros(2 * slots, np.int32)
    idx = rng.integers(0, slots, 60)
    ht1[2 * idx] = rng.integers(1, 50, 60)
    ht1[2 * idx + 1] = rng.integers(0, 9, 60)
    filters = [dict(col=f0, mode=1, c1=3, c2=15), dict(col=f1, mode=2, c1=-1, c2=4)]
    probes = [dict(fkey=k0, ht=ht0, num_slots=slots, layout=0),
              dict(fkey=k1, ht=ht1, num_slots=slots, layout=1, min_val=0, unique_val=1, res_slot=0)]
    for agg_op in (0, 1, 2):
        exp_scalar, _ = _py_star(n, filters, probes, [a0, a1], agg_op, 1, 0)
        res = np.zeros(1, np.uint64)
        st = O.star(n, filters=filters, probes=probes, aggr=[a0, a1], agg_op=agg_op, res_layout=0, res=res)
        assert st & 0x1  # keys below key_min are reported as probe-range errors
        assert int(res[0]) == exp_scalar
        _, exp_groups = _py_star(n, filters, probes, [a0, a1], agg_op, 9, 3)
        dense = np.zeros(9, np.int64)
        O.star(n, filters=filters, probes=probes, aggr=[a0, a1], agg_op=agg_op, total_val=9, res_layout=3,
               res=dense)
        assert {g: int(dense[g]) for g in exp_groups} == exp_groups


def test_merge_known_answer():
    cpu = np.zeros(12, np.int32)
    gpu = np.zeros(12, np.int32)
    cpu[0:2] = [1993, 7]
    cpu[4:6] = np.array([5], np.int64).view(np.int32)
    gpu[0:4] = [1993, 7, 0, 3]
    gpu[4:6] = np.array([-9], np.int64).view(np.int32)
    gpu[6:8] = [1994, 2]
    gpu[10:12] = np.array([11], np.int64).view(np.int32)
    O.merge(cpu, gpu, 2)
    assert list(cpu[0:4]) == [1993, 7, 0, 3] and list(cpu[6:10]) == [1994, 2, 0, 0]
    assert cpu[4:6].view(np.int64)[0] == -4 and cpu[10:12].view(np.int64)[0] == 11


def test_generator_calendar_and_ranges():
    s = ssb.Sizes(lo_len=100_000, s_len=1000, c_len=2000, p_len=3000)
    t = ssb.gen_host(s, 5, ALL_FACT, ALL_DIMS + ["d_yearmonthnum", "s_city", "s_nation", "c_city"])
    day0 = dt.date(1992, 1, 1)
    cal = [int((day0 + dt.timedelta(days=i)).strftime("%Y%m%d")) for i in range(2557)]
    assert list(t["d_datekey"]) == cal and cal[-1] == 19981231
    assert list(t["d_year"]) == [c // 10000 for c in cal]
    assert list(t["d_yearmonthnum"]) == [c // 100 for c in cal]
    assert set(np.unique(t["lo_orderdate"])) <= set(cal)
    assert t["lo_quantity"].min() >= 1 and t["lo_quantity"].max() <= 50
    assert t["lo_discount"].min() == 0 and t["lo_discount"].max() == 10
    assert t["lo_extendedprice"].min() >= 90100 and t["lo_extendedprice"].max() <= 10494950
    assert t["lo_supplycost"].min() >= 54000 and t["lo_supplycost"].max() <= 600000
    assert t["lo_suppkey"].min() >= 1 and t["lo_suppkey"].max() <= 1000
    assert list(t["s_suppkey"]) == list(range(1, 1001))
    assert np.array_equal(t["s_nation"], t["s_city"] // 10) and np.array_equal(t["s_region"], t["s_nation"] // 5)
    assert np.array_equal(t["p_category"], t["p_brand1"] // 40) and np.array_equal(t["p_mfgr"], t["p_category"] // 5)
    # determinism and independence from the thread count
    t2 = ssb.gen_host(s, 5, ["lo_orderdate"], [], nthreads=1)
    assert np.array_equal(t2["lo_orderdate"], t["lo_orderdate"])


def test_generator_restated_in_python():
    # splitmix64-based stream restated independently in Python ints
    M = 2**64 - 1

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    def uniform(seed, stream, row, lo, hi):
        base = mix((seed + 0x9E3779B97F4A7C15 * (stream + 1)) & M)
        r = mix((base + 0xD1B54A32D192ED03 * (row + 1)) & M) >> 32
        return lo + ((r * (hi - lo + 1)) >> 32)

    s = ssb.Sizes(lo_len=64, s_len=40000)
    t = ssb.gen_host(s, 123, ["lo_quantity", "lo_suppkey", "lo_revenue"], [])
    assert [int(x) for x in t["lo_quantity"]] == [uniform(123, 1, i, 1, 50) for i in range(64)]
    assert [int(x) for x in t["lo_suppkey"]] == [uniform(123, 4, i, 1, 40000) for i in range(64)]
    assert [int(x) for x in t["lo_revenue"]] == [uniform(123, 7, i, 90100, 10494950) for i in range(64)]
