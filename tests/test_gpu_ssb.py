"""GPU parity: every CUDA query path against the CPU oracle, bit for bit."""
import ctypes as C

import numpy as np
import pytest
import torch

from mordred_b200 import _lib as L
from mordred_b200 import ssb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SEG = 1 << 20
U64 = 2**64


@pytest.fixture(scope="module", autouse=True)
def device():
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    yield
    torch.cuda.synchronize()


def host(t):
    return {k: v.cpu().numpy() for k, v in t.items()}


def status():
    return L.device_status(0, clear=True)


# ---- filter-aggregate (q11 form) ---------------------------------------------------------

@pytest.mark.parametrize("n", [0, 1, 5, 2047, 2048, 2049, 8191, 196_625, 1_000_003, 6_000_000])
def test_q11_parity(n):
    s = ssb.Sizes(lo_len=n)
    t = ssb.gen_device(s, 100 + n, ssb.Q11_COLUMNS, [])
    ws_rev = torch.zeros(1, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("mb_q11_query", ssb._p(t["lo_orderdate"]), ssb._p(t["lo_discount"]), ssb._p(t["lo_quantity"]),
           ssb._p(t["lo_extendedprice"]), n, ssb._p(ws_rev), ssb._p(cnt), ssb._stream())
    torch.cuda.synchronize()
    h = host(t)
    assert int(ws_rev.item()) % U64 == O.q11(h)
    exp_cnt = int(np.count_nonzero((h["lo_discount"] >= 1) & (h["lo_discount"] <= 3) & (h["lo_quantity"] < 25)))
    assert int(cnt.item()) == exp_cnt
    assert status() == 0


def test_q11_full_size_and_repeat():
    n = 6_000_000
    t = ssb.gen_device(ssb.Sizes(lo_len=n), 2024, ssb.Q11_COLUMNS, [])
    rev = ssb.q11(t, n)
    first = int(rev.item())
    for _ in range(3):
        rev = ssb.q11(t, n)
        assert int(rev.item()) == first
    assert first % U64 == O.q11(host(t))
    assert status() == 0


# ---- Query A / Query B ---------------------------------------------------------------------

def _sizes(n, small):
    return ssb.Sizes(lo_len=n, s_len=2_000, c_len=30_000, p_len=20_000) if small else ssb.Sizes(lo_len=n)


@pytest.mark.parametrize("n,small", [(0, True), (1, True), (777, True), (2048 * 3 + 5, True), (500_000, True),
                                     (3_000_001, False)])
def test_query_a_parity(n, small):
    s = _sizes(n, small)
    t = ssb.gen_device(s, 7 + n, ssb.QA_FACT, ssb.QA_DIMS)
    ws = ssb.StarWorkspace(s)
    res = ssb.query_a(t, ws).cpu().numpy()
    h = host(t)
    exp, st = O.q21(h, ssb.DATE_SLOTS)
    assert st == 0 and status() == 0
    assert ssb.crystal4_groups(res) == O.q21_groups(exp)
    # raw result array, keys included, equals the oracle's pipeline in the same layout
    s_ht = ws["ht_s"].cpu().numpy()
    p_ht = ws["ht_p_a"].cpu().numpy()
    d_ht = ws["ht_d"].cpu().numpy()
    ref = np.zeros(4 * ssb.QA_GROUPS, np.int32)
    O.star(n, probes=[dict(fkey=h["lo_suppkey"], ht=s_ht, num_slots=s.s_len, layout=0),
                      dict(fkey=h["lo_partkey"], ht=p_ht, num_slots=s.p_len, layout=1, unique_val=7, res_slot=1),
                      dict(fkey=h["lo_orderdate"], ht=d_ht, num_slots=ssb.DATE_SLOTS, key_min=19920101, layout=1,
                           min_val=1992, unique_val=1, res_slot=0)],
           aggr=[h["lo_revenue"]], total_val=ssb.QA_GROUPS, res_layout=2, res=ref)
    assert np.array_equal(res, ref)


@pytest.mark.parametrize("n,small", [(0, True), (3, True), (4099, True), (500_000, True), (2_500_007, False)])
def test_query_b_parity(n, small):
    s = _sizes(n, small)
    t = ssb.gen_device(s, 41 + n, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    res = ssb.query_b(t, ws).cpu().numpy()
    exp, st = O.q41(host(t), ssb.DATE_SLOTS)
    assert st == 0 and status() == 0
    assert np.array_equal(res, exp)  # same int[4*175] layout, bit for bit


@pytest.mark.parametrize("region,category,mfgr", [(0, 0, (2, 3)), (4, 24, (4, 4)), (2, 13, (1, 3))])
def test_query_constants(region, category, mfgr):
    s = ssb.Sizes(lo_len=400_000, s_len=5_000, c_len=50_000, p_len=80_000)
    t = ssb.gen_device(s, 99, sorted(set(ssb.QA_FACT + ssb.QB_FACT)), sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    h = host(t)
    ra = ssb.query_a(t, ws, category=category, region=region).cpu().numpy()
    assert ssb.crystal4_groups(ra) == O.q21_groups(O.q21(h, ssb.DATE_SLOTS, category=category, region=region)[0])
    rb = ssb.query_b(t, ws, c_region=region, s_region=(region + 1) % 5, mfgr=mfgr).cpu().numpy()
    eb, _ = O.q41(h, ssb.DATE_SLOTS, c_region=region, s_region=(region + 1) % 5, mfgr=mfgr)
    assert np.array_equal(rb, eb)


def test_full_size_star_queries():
    """Query A and Query B at 120,000,000 fact rows, bit-exact against the oracle."""
    s = ssb.Sizes(lo_len=120_000_000)
    t = ssb.gen_device(s, 2026, ssb.QB_FACT, sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    ra = ssb.query_a(t, ws).cpu().numpy()
    rb = ssb.query_b(t, ws).cpu().numpy()
    assert status() == 0
    h = host(t)
    del t
    torch.cuda.empty_cache()
    assert ssb.crystal4_groups(ra) == O.q21_groups(O.q21(h, ssb.DATE_SLOTS)[0])
    assert np.array_equal(rb, O.q41(h, ssb.DATE_SLOTS)[0])
    dense = ssb.query_a_dense(ra)
    assert dense.shape == (7, 1000) and int(dense.sum()) == sum(g[2] for g in ssb.crystal4_groups(ra))


def test_determinism_and_accumulation():
    s = ssb.Sizes(lo_len=1_234_567, s_len=3_000, c_len=40_000, p_len=60_000)
    t = ssb.gen_device(s, 5, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    r1 = ssb.query_b(t, ws).cpu().numpy().copy()
    r2 = ssb.query_b(t, ws).cpu().numpy().copy()
    assert np.array_equal(r1, r2)
    # a second probe call without zeroing accumulates (caller-owned result, as the reference)
    L.call("mb_q41_probe", *[ssb._p(t[k]) for k in ("lo_orderdate", "lo_partkey", "lo_custkey", "lo_suppkey",
                                                     "lo_revenue", "lo_supplycost")], s.lo_len,
           ssb._p(ws["ht_p_b"]), s.p_len, ssb._p(ws["ht_s"]), s.s_len, ssb._p(ws["ht_c"]), s.c_len,
           ssb._p(ws["ht_d"]), ssb.DATE_SLOTS, ssb._p(ws["res_b"]), ssb._stream())
    r3 = ws["res_b"].cpu().numpy().reshape(-1, 4)
    s1 = r1.reshape(-1, 4)[:, 2:4].copy().view(np.int64)
    s3 = r3[:, 2:4].copy().view(np.int64)
    assert np.array_equal(s3, 2 * s1)


# ---- builds --------------------------------------------------------------------------------

def test_pht_builds_bit_identical():
    s = ssb.Sizes(lo_len=0, s_len=40_000, c_len=600_000, p_len=1_000_000)
    t = ssb.gen_device(s, 3, [], ["s_suppkey", "s_region", "p_partkey", "p_brand1", "p_mfgr", "d_datekey", "d_year"])
    h = host(t)
    st = ssb._stream()
    # KEY layout with a filter and a presence bitmap
    ht = torch.zeros(s.s_len, dtype=torch.int32, device="cuda")
    bm = torch.zeros((s.s_len + 31) // 32, dtype=torch.int32, device="cuda")
    L.call("mb_build_pht", ssb._p(t["s_region"]), L.MB_FILTER_EQ, 2, 0, ssb._p(t["s_suppkey"]), None, s.s_len,
           ssb._p(ht), s.s_len, 0, ssb._p(bm), st)
    ref = np.zeros(s.s_len, np.int32)
    refbm = np.zeros((s.s_len + 31) // 32, np.uint32)
    O.build_ht(h["s_region"], 0, 2, 0, h["s_suppkey"], None, ref, s.s_len, 0, 0, presence=refbm)
    assert np.array_equal(ht.cpu().numpy(), ref)
    assert np.array_equal(bm.cpu().numpy().view(np.uint32), refbm)
    # KEY_VAL layout, EQ OR EQ filter
    ht2 = torch.zeros(2 * s.p_len, dtype=torch.int32, device="cuda")
    L.call("mb_build_pht", ssb._p(t["p_mfgr"]), L.MB_FILTER_EQ_OR_EQ, 1, 3, ssb._p(t["p_partkey"]),
           ssb._p(t["p_brand1"]), s.p_len, ssb._p(ht2), s.p_len, 0, None, st)
    ref2 = np.zeros(2 * s.p_len, np.int32)
    O.build_ht(h["p_mfgr"], 2, 1, 3, h["p_partkey"], h["p_brand1"], ref2, s.p_len, 0, 1)
    assert np.array_equal(ht2.cpu().numpy(), ref2)
    # date table with key_min, BETWEEN filter on the key itself
    ht3 = torch.zeros(2 * ssb.DATE_SLOTS, dtype=torch.int32, device="cuda")
    L.call("mb_build_pht", ssb._p(t["d_datekey"]), L.MB_FILTER_BETWEEN, 19940101, 19961231,
           ssb._p(t["d_datekey"]), ssb._p(t["d_year"]), s.d_len, ssb._p(ht3), ssb.DATE_SLOTS, 19920101, None, st)
    ref3 = np.zeros(2 * ssb.DATE_SLOTS, np.int32)
    O.build_ht(h["d_datekey"], 1, 19940101, 19961231, h["d_datekey"], h["d_year"], ref3, ssb.DATE_SLOTS,
               19920101, 1)
    assert np.array_equal(ht3.cpu().numpy(), ref3)
    assert status() == 0


@pytest.mark.parametrize("n_dim", [50_000, 100_000])
def test_src_ops_join(n_dim):
    """src/ops join at two table sizes: 100,000 slots are probed in L2; 50,000 get a
    presence bitmap that the dense phase tests, and the payload is read afterwards."""
    n_fact = 3_000_011
    g = torch.Generator(device="cpu").manual_seed(1)
    dim_key = torch.randperm(n_dim, generator=g).to(torch.int32) + 1
    dim_val = torch.randint(-5000, 5000, (n_dim,), generator=g, dtype=torch.int32)
    fkey = torch.randint(1, n_dim + 1, (n_fact,), generator=g, dtype=torch.int32)
    fval = torch.randint(-(2**20), 2**20, (n_fact,), generator=g, dtype=torch.int32)
    d = {k: v.cuda() for k, v in dict(dim_key=dim_key, dim_val=dim_val, fkey=fkey, fval=fval).items()}
    ht = torch.zeros(2 * n_dim, dtype=torch.int32, device="cuda")
    res = torch.zeros(1, dtype=torch.int64, device="cuda")
    L.call("mb_join_build", ssb._p(d["dim_key"]), ssb._p(d["dim_val"]), n_dim, ssb._p(ht), n_dim, ssb._stream())
    L.call("mb_join_probe", ssb._p(d["fkey"]), ssb._p(d["fval"]), n_fact, ssb._p(ht), n_dim, ssb._p(res),
           ssb._stream())
    lookup = np.zeros(n_dim + 1, np.int64)
    lookup[dim_key.numpy()] = dim_val.numpy()
    prod = (fval.numpy().astype(np.int64) * lookup[fkey.numpy()])
    prod = ((prod + 2**31) % 2**32) - 2**31  # int32 product (src/ops/join.cu:73)
    assert int(res.item()) % U64 == int(prod.sum()) % U64


# ---- generic pipeline: variants, alignment, status ------------------------------------------

def _qb_args(t, ws, s, res, **kw):
    return ssb.star_args(
        num_rows=kw.pop("n", s.lo_len),
        probes=[dict(fkey=t["lo_suppkey"], ht=ws["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
                dict(fkey=t["lo_custkey"], ht=ws["ht_c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
                     res_slot=1),
                dict(fkey=t["lo_partkey"], ht=ws["ht_p_b"], num_slots=s.p_len, layout=L.MB_HT_KEY),
                dict(fkey=t["lo_orderdate"], ht=ws["ht_d"], num_slots=ssb.DATE_SLOTS, key_min=19920101,
                     layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)],
        aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=ssb.QB_GROUPS,
        res_layout=L.MB_RES_CRYSTAL4, res=res, **kw)


def test_launch_variants_identical():
    s = ssb.Sizes(lo_len=2_000_003, s_len=4_000, c_len=50_000, p_len=70_000)
    t = ssb.gen_device(s, 17, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    base = ssb.query_b(t, ws).cpu().numpy().copy()
    for threads in (128, 256, 512, 640, 768):
        for ipt in (4, 8, 16):
            for stages in (2, 3, 6):
                if (threads == 512 and ipt == 16) or (threads > 512 and ipt != 8):
                    continue  # 20 and 24 consumer warps: 8 rows a thread only
                res = torch.zeros(4 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
                ssb.star_query(_qb_args(t, ws, s, res, threads=threads, items_per_thread=ipt, stages=stages))
                assert np.array_equal(res.cpu().numpy(), base), (threads, ipt, stages)
    for grid in (1, 7, 148 * 3):
        res = torch.zeros(4 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
        ssb.star_query(_qb_args(t, ws, s, res, grid=grid))
        assert np.array_equal(res.cpu().numpy(), base), grid
    assert status() == 0


def test_misaligned_columns_take_the_plain_path():
    s = ssb.Sizes(lo_len=1_000_001, s_len=4_000, c_len=50_000, p_len=70_000)
    t = ssb.gen_device(s, 23, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    ssb.query_b(t, ws)
    shifted = {k: (v[1:] if k.startswith("lo_") else v) for k, v in t.items()}
    res = torch.zeros(4 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
    ssb.star_query(_qb_args(shifted, ws, s, res, n=s.lo_len - 1))
    h = host(shifted)
    exp, _ = O.q41(h, ssb.DATE_SLOTS)
    assert np.array_equal(res.cpu().numpy(), exp)


def test_probe_and_group_range_are_reported():
    n = 100_000
    rng = np.random.default_rng(0)
    key = rng.integers(-50, 500, n).astype(np.int32)
    val = rng.integers(-100, 100, n).astype(np.int32)
    ht = np.zeros(2 * 400, np.int32)
    ht[0::2] = np.arange(1, 401)
    ht[1::2] = rng.integers(-3, 20, 400)      # negative payloads make negative group indexes
    dk, dv, dht = (torch.from_numpy(x).cuda() for x in (key, val, ht))
    res = torch.zeros(16, dtype=torch.int64, device="cuda")
    a = ssb.star_args(num_rows=n, probes=[dict(fkey=dk, ht=dht, num_slots=400, layout=L.MB_HT_KEY_VAL,
                                               unique_val=1)],
                      aggr=[dv], agg_op=L.MB_AGG_SUM, total_val=16, res_layout=L.MB_RES_DENSE, res=res)
    ssb.star_query(a)
    st = status()
    exp = np.zeros(16, np.int64)
    ost = O.star(n, probes=[dict(fkey=key, ht=ht, num_slots=400, layout=1, unique_val=1)], aggr=[val], agg_op=0,
                 total_val=16, res_layout=3, res=exp)
    assert st == ost == (L.MB_STATUS_PROBE_RANGE | L.MB_STATUS_GROUP_RANGE)
    assert np.array_equal(res.cpu().numpy(), exp)


def test_filters_and_count():
    n = 3_333_333
    s = ssb.Sizes(lo_len=n)
    t = ssb.gen_device(s, 77, ["lo_orderdate", "lo_quantity", "lo_discount", "lo_extendedprice"], [])
    h = host(t)
    for modes in [(L.MB_FILTER_EQ, 5, 0), (L.MB_FILTER_EQ_OR_EQ, 3, 7), (L.MB_FILTER_BETWEEN, 2, 8)]:
        for count_after in (-1, 0, 1, 2):
            res = torch.zeros(1, dtype=torch.int64, device="cuda")
            cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
            filters = [dict(col=t["lo_discount"], mode=modes[0], c1=modes[1], c2=modes[2]),
                       dict(col=t["lo_orderdate"], mode=L.MB_FILTER_BETWEEN, c1=19950101, c2=19971231)]
            ssb.star_query(ssb.star_args(num_rows=n, filters=filters, aggr=[t["lo_extendedprice"], t["lo_quantity"]],
                                         agg_op=L.MB_AGG_MUL, res_layout=L.MB_RES_SCALAR, res=res, count=cnt,
                                         count_after=count_after))
            exp = np.zeros(1, np.uint64)
            ecnt = np.zeros(1, np.uint64)
            hf = [dict(col=h["lo_discount"], mode=modes[0], c1=modes[1], c2=modes[2]),
                  dict(col=h["lo_orderdate"], mode=1, c1=19950101, c2=19971231)]
            O.star(n, filters=hf, aggr=[h["lo_extendedprice"], h["lo_quantity"]], agg_op=2, res_layout=0, res=exp,
                   count=ecnt, count_after=count_after)
            assert int(res.item()) % U64 == int(exp[0])
            assert int(cnt.item()) == int(ecnt[0])


# ---- engine (segment-cache) entry points ------------------------------------------------------

def _engine_setup(seed=31, nseg=6, tail=12345):
    lo_len = (nseg - 1) * SEG + tail
    s = ssb.Sizes(lo_len=lo_len, s_len=8_000, c_len=90_000, p_len=150_000)
    fact = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate", "lo_revenue", "lo_supplycost", "lo_quantity"]
    t = ssb.gen_device(s, seed, fact, ssb.QB_DIMS)
    # scatter every fact segment of every column into a shuffled gpuCache
    rng = np.random.default_rng(seed)
    nslots = nseg * len(fact) + 3
    cache = torch.zeros(nslots * SEG, dtype=torch.int32, device="cuda")
    slots = rng.permutation(nslots)[: nseg * len(fact)].reshape(len(fact), nseg)
    col_idx = {}
    for ci, name in enumerate(fact):
        for sg in range(nseg):
            lo, hi = sg * SEG, min((sg + 1) * SEG, lo_len)
            cache[int(slots[ci, sg]) * SEG: int(slots[ci, sg]) * SEG + (hi - lo)] = t[name][lo:hi]
        col_idx[name] = torch.from_numpy(slots[ci].astype(np.int32)).cuda()
    return s, t, cache, col_idx, nseg, lo_len


def _engine_hts(t, s):
    """Engine-layout HTs via mb_build_GPU2 (direct columns) and the same on the CPU."""
    h = host(t)
    specs = [("s", "s_suppkey", None, "s_region", 1, 1, 1, s.s_len, 0),
             ("c", "c_custkey", "c_nation", "c_region", 1, 1, 1, s.c_len, 0),
             ("p", "p_partkey", None, "p_mfgr", 2, 0, 1, s.p_len, 0),
             ("d", "d_datekey", "d_year", None, 0, 0, 0, ssb.DATE_SLOTS, 19920101)]
    out = {}
    for name, key, val, flt, mode, c1, c2, slots, kmin in specs:
        ht = torch.zeros(2 * slots, dtype=torch.int32, device="cuda")
        f = L.MbFilterArgsGPU(ssb._p(t[flt]) if flt else None, None, c1, c2, 0, 0, mode, 0)
        b = L.MbBuildArgsGPU(ssb._p(t[key]), ssb._p(t[val]) if val else None, slots, kmin, 0)
        L.call("mb_build_GPU2", None, C.byref(f), C.byref(b), len(h[key]), ssb._p(ht), 0, None, ssb._stream())
        ref = np.zeros(2 * slots, np.int32)
        O.build_ht(h[flt] if flt else None, mode, c1, c2, h[key], h[val] if val else None, ref, slots, kmin, 2)
        assert np.array_equal(ht.cpu().numpy(), ref), name
        out[name] = (ht, ref, slots, kmin)
    return out


@pytest.mark.parametrize("segments", [None, [3, 0, 1, 5], [5], [2, 4], [4, 0, 2, 3, 1, 5]])
def test_engine_filter_probe_group_by_segment_cache(segments):
    s, t, cache, col_idx, nseg, lo_len = _engine_setup()
    hts = _engine_hts(t, s)
    h = host(t)
    if segments is None:
        seg_arr, num_tuples, start = None, lo_len, 0
    else:
        seg_arr = np.array(segments, np.int16)
        last = nseg - 1
        num_tuples = sum(SEG if sg != last else lo_len - last * SEG for sg in segments)
        assert segments[-1] == last or all(sg != last for sg in segments)
        start = 0
    f = L.MbFilterArgsGPU(ssb._p(col_idx["lo_quantity"]), ssb._p(col_idx["lo_orderdate"]), 5, 40, 19930601, 19970630,
                          1, 1)
    p = L.MbProbeArgsGPU(*(ssb._p(col_idx[k]) for k in ("lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate")),
                         *(ssb._p(hts[k][0]) for k in "scpd"), *(hts[k][2] for k in "scpd"),
                         *(hts[k][3] for k in "scpd"))
    g = L.MbGroupbyArgsGPU(ssb._p(col_idx["lo_revenue"]), ssb._p(col_idx["lo_supplycost"]), None, None, None, None,
                           0, 0, 0, 1992, 0, 7, 0, 1, ssb.QB_GROUPS, 0)
    res = torch.zeros(6 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
    seg_dev = torch.from_numpy(seg_arr).cuda() if seg_arr is not None else None
    L.call("mb_filter_probe_group_by_GPU2", ssb._p(cache), C.byref(f), C.byref(p), C.byref(g), num_tuples,
           ssb._p(res), start, ssb._p(seg_dev), ssb._stream())
    exp = np.zeros(6 * ssb.QB_GROUPS, np.int32)
    probes = []
    for slot, (k, fk, mn, uq) in enumerate([("s", "lo_suppkey", 0, 0), ("c", "lo_custkey", 0, 7),
                                             ("p", "lo_partkey", 0, 0), ("d", "lo_orderdate", 1992, 1)]):
        probes.append(dict(fkey=h[fk], ht=hts[k][1], num_slots=hts[k][2], key_min=hts[k][3], layout=2, min_val=mn,
                           unique_val=uq, res_slot=slot))
    ost = O.star(num_tuples, filters=[dict(col=h["lo_quantity"], mode=1, c1=5, c2=40),
                                      dict(col=h["lo_orderdate"], mode=1, c1=19930601, c2=19970630)],
                 probes=probes, aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=ssb.QB_GROUPS,
                 res_layout=1, res=exp, segment_group=seg_arr, start_offset=start, segment_size=SEG)
    assert ost == 0 and status() == 0
    assert np.array_equal(res.cpu().numpy(), exp)


def test_engine_probe_group_by_and_aggr():
    s, t, cache, col_idx, nseg, lo_len = _engine_setup(seed=5, nseg=3, tail=777)
    hts = _engine_hts(t, s)
    h = host(t)
    # probe_group_by_GPU2: supplier + date only, group by year; the absent slots add their (0 - min) * unique
    p = L.MbProbeArgsGPU(ssb._p(col_idx["lo_suppkey"]), None, None, ssb._p(col_idx["lo_orderdate"]),
                         ssb._p(hts["s"][0]), None, None, ssb._p(hts["d"][0]), hts["s"][2], 0, 0, hts["d"][2],
                         0, 0, 0, 19920101)
    g = L.MbGroupbyArgsGPU(ssb._p(col_idx["lo_revenue"]), None, None, None, None, None, 0, 0, -3, 1992, 0, 0, 2, 1,
                           7 + 6, 0)
    res = torch.zeros(6 * 13, dtype=torch.int32, device="cuda")
    L.call("mb_probe_group_by_GPU2", ssb._p(cache), C.byref(p), C.byref(g), lo_len, ssb._p(res), 0, None,
           ssb._stream())
    exp = np.zeros(6 * 13, np.int32)
    O.star(lo_len, probes=[dict(fkey=h["lo_suppkey"], ht=hts["s"][1], num_slots=hts["s"][2], layout=2, res_slot=0),
                           dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=hts["d"][2], key_min=19920101,
                                layout=2, min_val=1992, unique_val=1, res_slot=3)],
           aggr=[h["lo_revenue"]], agg_op=0, total_val=13, group_bias=(0 + 3) * 2, res_layout=1, res=exp,
           segment_size=SEG)
    assert np.array_equal(res.cpu().numpy(), exp)
    # filter_probe_aggr_GPU2: date probe only, SUM(revenue * quantity-like column) into res[4]
    f = L.MbFilterArgsGPU(ssb._p(col_idx["lo_quantity"]), None, 1, 24, 0, 0, 1, 0)
    g2 = L.MbGroupbyArgsGPU(ssb._p(col_idx["lo_revenue"]), ssb._p(col_idx["lo_quantity"]), None, None, None, None,
                            0, 0, 0, 0, 0, 0, 0, 0, 1, 1)
    res2 = torch.zeros(6, dtype=torch.int32, device="cuda")
    L.call("mb_filter_probe_aggr_GPU2", ssb._p(cache), C.byref(f), C.byref(p), C.byref(g2), lo_len, ssb._p(res2), 0,
           None, ssb._stream())
    exp2 = np.zeros(1, np.uint64)
    O.star(lo_len, filters=[dict(col=h["lo_quantity"], mode=1, c1=1, c2=24)],
           probes=[dict(fkey=h["lo_orderdate"], ht=hts["d"][1], num_slots=hts["d"][2], key_min=19920101, layout=2)],
           aggr=[h["lo_revenue"], h["lo_quantity"]], agg_op=2, res_layout=0, res=exp2, segment_size=SEG)
    got = res2.cpu().numpy()[4:6].view(np.uint64)[0]
    assert int(got) == int(exp2[0])
    assert status() == 0


def test_engine_build_segment_cache():
    """build_GPU2 over a dimension split across two cache segments; row ids are table positions."""
    n = SEG + 4321
    s = ssb.Sizes(lo_len=0, p_len=n)
    t = ssb.gen_device(s, 8, [], ["p_partkey", "p_brand1", "p_category"])
    h = host(t)
    cache = torch.zeros(6 * SEG, dtype=torch.int32, device="cuda")
    slots = {"p_partkey": [3, 1], "p_brand1": [0, 4], "p_category": [2, 5]}
    for name, sl in slots.items():
        for sg, slot in enumerate(sl):
            lo, hi = sg * SEG, min((sg + 1) * SEG, n)
            cache[slot * SEG: slot * SEG + (hi - lo)] = t[name][lo:hi]
    col = {k: torch.tensor(v, dtype=torch.int32, device="cuda") for k, v in slots.items()}
    ht = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    f = L.MbFilterArgsGPU(ssb._p(col["p_category"]), None, 3, 9, 0, 0, 1, 0)
    b = L.MbBuildArgsGPU(ssb._p(col["p_partkey"]), ssb._p(col["p_brand1"]), n, 0, 0)
    L.call("mb_build_GPU2", ssb._p(cache), C.byref(f), C.byref(b), n, ssb._p(ht), 0, None, ssb._stream())
    ref = np.zeros(2 * n, np.int32)
    O.build_ht(h["p_category"], 1, 3, 9, h["p_partkey"], h["p_brand1"], ref, n, 0, 2)
    assert np.array_equal(ht.cpu().numpy(), ref)
    assert status() == 0
