"""Cluster-resident mirrors of the sparse phase's hash tables (mb_star_args.mirrors): the
star kernel with mirrors on equals the oracle (and the kernel with mirrors off) for the
Query A / Query B shapes, the engine four-table shapes over direct columns and over the
segment cache, payload codes that overflow their 4 bits, and every launch shape that has
a mirror variant."""
import numpy as np
import pytest

from mordred_b200 import _lib as L
from mordred_b200 import ssb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SEG = 1 << 20


@pytest.fixture(scope="module", autouse=True)
def device():
    import torch
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    yield
    torch.cuda.synchronize()


def _tables(n, seed, s_len=40_000, c_len=600_000, p_len=1_000_000):
    s = ssb.Sizes(lo_len=n, s_len=s_len, c_len=c_len, p_len=p_len)
    t = ssb.gen_device(s, seed, ssb.QB_FACT, sorted(set(ssb.QA_DIMS + ssb.QB_DIMS + ["s_nation"])))
    return s, t, {k: v.cpu().numpy() for k, v in t.items()}


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _run(probes, t, n, aggr, agg_op, total, layout, mirrors, threads, items, **extra):
    import torch
    res = torch.zeros(4 * total if layout == L.MB_RES_CRYSTAL4 else 6 * total, dtype=torch.int32, device="cuda")
    a = ssb.star_args(num_rows=n, probes=probes, aggr=aggr, agg_op=agg_op, total_val=total, res_layout=layout,
                      res=res, mirrors=mirrors, threads=threads, items_per_thread=items, **extra)
    ssb.star_query(a)
    return res.cpu().numpy()


@pytest.mark.parametrize("threads,items", [(256, 8), (512, 8), (256, 16)])
@pytest.mark.parametrize("date_min", [1992, 1984])
def test_query_b_shape_with_mirrors(threads, items, date_min):
    """supplier bitmap -> customer (presence bits, nation read for survivors) -> part
    (presence bits) -> date (4-bit year codes; with date_min 1984 the year 1998 does not
    fit a code and is read from the table)."""
    n = 9_000_011
    s, t, h = _tables(n, 77)
    ht = {}
    for name, flt, mode, c1, c2, key, val, slots, kmin, lay in [
            ("s", "s_region", 0, 1, 0, "s_suppkey", None, s.s_len, 0, 0),
            ("c", "c_region", 0, 1, 0, "c_custkey", "c_nation", s.c_len, 0, 1),
            ("p", "p_mfgr", 2, 0, 1, "p_partkey", None, s.p_len, 0, 0),
            ("d", None, 0, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN, 1)]:
        a = np.zeros(2 * slots if lay else slots, np.int32)
        O.build_ht(h[flt] if flt else None, mode, c1, c2, h[key], h[val] if val else None, a, slots, kmin, lay)
        ht[name] = (a, _dev(a))
    # group nation * uc + (year - date_min): one key tuple per group either way; with
    # date_min 1984 the years give 8..14, so the code of 1998 escapes
    uc, total = (7, 175) if date_min == 1992 else (14, 25 * 14 + 15)
    probes = lambda d: [dict(fkey=d["lo_suppkey"], ht=ht["s"][1 if d is t else 0], num_slots=s.s_len, layout=0),
                        dict(fkey=d["lo_custkey"], ht=ht["c"][1 if d is t else 0], num_slots=s.c_len, layout=1,
                             unique_val=uc, res_slot=1),
                        dict(fkey=d["lo_partkey"], ht=ht["p"][1 if d is t else 0], num_slots=s.p_len, layout=0),
                        dict(fkey=d["lo_orderdate"], ht=ht["d"][1 if d is t else 0], num_slots=ssb.DATE_SLOTS,
                             key_min=ssb.DATE_MIN, layout=1, min_val=date_min, unique_val=1, res_slot=0)]
    exp = np.zeros(4 * total, np.int32)
    assert O.star(n, probes=probes(h), aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=total,
                  res_layout=2, res=exp) == 0
    for mirrors in (2, 1):
        got = _run(probes(t), t, n, [t["lo_revenue"], t["lo_supplycost"]], L.MB_AGG_SUB, total, L.MB_RES_CRYSTAL4,
                   mirrors, threads, items)
        assert np.array_equal(got, exp), (mirrors, threads, items, date_min)
    assert L.device_status(0, clear=True) == 0


@pytest.mark.parametrize("threads,items", [(256, 8), (512, 8)])
def test_query_a_shape_with_mirrors(threads, items):
    """supplier bitmap -> part (presence bits, brand read for survivors) -> date (codes)."""
    n = 8_400_007
    s, t, h = _tables(n, 5)
    ht = {}
    for name, flt, c1, key, val, slots, kmin, lay in [("s", "s_region", 2, "s_suppkey", None, s.s_len, 0, 0),
                                                       ("p", "p_category", 3, "p_partkey", "p_brand1", s.p_len, 0, 1),
                                                       ("d", None, 0, "d_datekey", "d_year", ssb.DATE_SLOTS,
                                                        ssb.DATE_MIN, 1)]:
        a = np.zeros(2 * slots if lay else slots, np.int32)
        O.build_ht(h[flt] if flt else None, 0, c1, 0, h[key], h[val] if val else None, a, slots, kmin, lay)
        ht[name] = (a, _dev(a))
    probes = lambda d, k: [dict(fkey=d["lo_suppkey"], ht=ht["s"][k], num_slots=s.s_len, layout=0),
                           dict(fkey=d["lo_partkey"], ht=ht["p"][k], num_slots=s.p_len, layout=1, unique_val=7,
                                res_slot=1),
                           dict(fkey=d["lo_orderdate"], ht=ht["d"][k], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                                layout=1, min_val=1992, unique_val=1, res_slot=0)]
    exp = np.zeros(4 * ssb.QA_GROUPS, np.int32)
    assert O.star(n, probes=probes(h, 0), aggr=[h["lo_revenue"]], agg_op=0, total_val=ssb.QA_GROUPS, res_layout=2,
                  res=exp) == 0
    for mirrors in (2, 1):
        got = _run(probes(t, 1), t, n, [t["lo_revenue"]], L.MB_AGG_SUM, ssb.QA_GROUPS, L.MB_RES_CRYSTAL4, mirrors,
                   threads, items)
        assert np.array_equal(got, exp), (mirrors, threads, items)
    # unpacked early stage return, 16 / 20 / 24 consumer warps, shared-memory and L2 groups
    for wide, group_mode in ((threads, 0), (640, 1), (768, 2), (768, 1)):
        got = _run(probes(t, 1), t, n, [t["lo_revenue"]], L.MB_AGG_SUM, ssb.QA_GROUPS, L.MB_RES_CRYSTAL4, 1,
                   wide, 8, pack=4, group_mode=group_mode)
        assert np.array_equal(got, exp), (wide, group_mode)
    assert L.device_status(0, clear=True) == 0


@pytest.mark.parametrize("cache", [False, True])
def test_engine_four_table_shape_with_mirrors(cache):
    """The engine's probe_group_by over VAL_OFF tables (group values read as payloads),
    grouped by (c_nation, year) with the supplier and part payloads unused, over direct
    columns and over a shuffled segment cache."""
    import torch
    nseg = 9
    n = (nseg - 1) * SEG + 4321
    s, t, h = _tables(n, 13, s_len=20_000, c_len=300_000, p_len=500_000)
    ht = {}
    for name, flt, mode, c1, c2, key, val, slots, kmin in [
            ("s", "s_region", 1, 0, 2, "s_suppkey", None, s.s_len, 0),
            ("c", "c_region", 0, 3, 0, "c_custkey", "c_nation", s.c_len, 0),
            ("p", "p_mfgr", 2, 1, 4, "p_partkey", None, s.p_len, 0),
            ("d", None, 0, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN)]:
        a = np.zeros(2 * slots, np.int32)
        O.build_ht(h[flt] if flt else None, mode, c1, c2, h[key], h[val] if val else None, a, slots, kmin, 2)
        ht[name] = (a, _dev(a))
    cols = {k: t[k] for k in ("lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue",
                              "lo_supplycost")}
    extra = {}
    if cache:
        rng = np.random.default_rng(3)
        names = list(cols)
        slots = rng.permutation(len(names) * nseg + 2)[: len(names) * nseg].reshape(len(names), nseg)
        pool = torch.zeros((len(names) * nseg + 2) * SEG, dtype=torch.int32, device="cuda")
        idx = {}
        for ci, name in enumerate(names):
            for sg in range(nseg):
                lo, hi = sg * SEG, min((sg + 1) * SEG, n)
                pool[int(slots[ci, sg]) * SEG: int(slots[ci, sg]) * SEG + (hi - lo)] = t[name][lo:hi]
            idx[name] = _dev(slots[ci].astype(np.int32))
        cols = idx
        extra = dict(gpu_cache=pool, segment_size=SEG)
    probes = lambda d, k: [dict(fkey=d["lo_suppkey"], ht=ht["s"][k], num_slots=s.s_len, layout=2),
                           dict(fkey=d["lo_custkey"], ht=ht["c"][k], num_slots=s.c_len, layout=2, unique_val=7,
                                res_slot=1),
                           dict(fkey=d["lo_partkey"], ht=ht["p"][k], num_slots=s.p_len, layout=2),
                           dict(fkey=d["lo_orderdate"], ht=ht["d"][k], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                                layout=2, min_val=1992, unique_val=1, res_slot=3)]
    exp = np.zeros(6 * 175, np.int32)
    assert O.star(n, probes=probes(h, 0), aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=175,
                  res_layout=1, res=exp) == 0
    for mirrors, threads, pack in ((2, 256, 0), (1, 256, 0), (1, 512, 3), (1, 768, 2), (1, 640, 3)):
        got = _run(probes(cols, 1), cols, n, [cols["lo_revenue"], cols["lo_supplycost"]], L.MB_AGG_SUB, 175,
                   L.MB_RES_ENGINE6, mirrors, threads, 8, pack=pack, **extra)
        assert np.array_equal(got, exp), (mirrors, threads, pack, cache)
    assert L.device_status(0, clear=True) == 0


@pytest.mark.parametrize("threads,items", [(256, 8), (512, 8), (256, 16), (640, 8), (768, 8)])
def test_packed_second_round_query_b_and_engine_shapes(threads, items):
    """The packed second sparse round (mb_star_args.pack = 2), the packed round that hands
    each stage back before its last batch of survivors is probed from registers (3) and
    the plain one (1) equal the oracle for the Query B shape (customer first), the same
    shape with every supplier present (several survivor batches per warp and tile) and
    the engine shape (supplier settled by its bitmap and read for its payload after the
    customer probe). 640 and 768 threads run 20 and 24 consumer warps over tiles of 16
    slices, handed out round robin."""
    n = 5_000_017
    s, t, h = _tables(n, 91, s_len=20_000, c_len=300_000, p_len=500_000)
    ht = {}
    for name, flt, mode, c1, c2, key, val, slots, kmin, lay in [
            ("s", "s_region", 0, 1, 0, "s_suppkey", None, s.s_len, 0, 0),
            ("s_all", None, 0, 0, 0, "s_suppkey", None, s.s_len, 0, 0),
            ("c", "c_region", 0, 1, 0, "c_custkey", "c_nation", s.c_len, 0, 1),
            ("p", "p_mfgr", 2, 0, 1, "p_partkey", None, s.p_len, 0, 0),
            ("d", None, 0, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN, 1),
            ("s2", "s_region", 1, 0, 2, "s_suppkey", "s_nation", s.s_len, 0, 2),
            ("c2", "c_region", 0, 3, 0, "c_custkey", "c_nation", s.c_len, 0, 2),
            ("p2", "p_mfgr", 2, 1, 4, "p_partkey", None, s.p_len, 0, 2),
            ("d2", None, 0, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN, 2)]:
        a = np.zeros(2 * slots if lay else slots, np.int32)
        O.build_ht(h[flt] if flt else None, mode, c1, c2, h[key], h[val] if val else None, a, slots, kmin, lay)
        ht[name] = (a, _dev(a))
    qb = lambda d, k, sup="s": [dict(fkey=d["lo_suppkey"], ht=ht[sup][k], num_slots=s.s_len, layout=0),
                       dict(fkey=d["lo_custkey"], ht=ht["c"][k], num_slots=s.c_len, layout=1, unique_val=7,
                            res_slot=1),
                       dict(fkey=d["lo_partkey"], ht=ht["p"][k], num_slots=s.p_len, layout=0),
                       dict(fkey=d["lo_orderdate"], ht=ht["d"][k], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                            layout=1, min_val=1992, unique_val=1, res_slot=0)]
    eng = lambda d, k: [dict(fkey=d["lo_suppkey"], ht=ht["s2"][k], num_slots=s.s_len, layout=2, unique_val=175,
                             res_slot=0),
                        dict(fkey=d["lo_custkey"], ht=ht["c2"][k], num_slots=s.c_len, layout=2, unique_val=7,
                             res_slot=1),
                        dict(fkey=d["lo_partkey"], ht=ht["p2"][k], num_slots=s.p_len, layout=2),
                        dict(fkey=d["lo_orderdate"], ht=ht["d2"][k], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                             layout=2, min_val=1992, unique_val=1, res_slot=3)]
    qb_all = lambda d, k: qb(d, k, "s_all")
    for probes, layout, total in ((qb, 2, 175), (qb_all, 2, 175), (eng, 1, 25 * 175)):
        exp = np.zeros((4 if layout == 2 else 6) * total, np.int32)
        assert O.star(n, probes=probes(h, 0), aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=total,
                      res_layout=layout, res=exp) == 0
        for pack in ((1, 2, 3) if threads <= 512 else (2, 3)):
            got = _run(probes(t, 1), t, n, [t["lo_revenue"], t["lo_supplycost"]], L.MB_AGG_SUB, total, layout, 1,
                       threads, items, pack=pack)
            assert np.array_equal(got, exp), (layout, pack, threads, items)
    assert L.device_status(0, clear=True) == 0
