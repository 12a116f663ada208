"""Selection with compaction (offset lists) on the GPU, and CPU/GPU split execution:
the GPU selects, the offset list crosses to the host, the CPU engine aggregates."""
import ctypes as C

import numpy as np
import pytest
import torch

from mordred_b200 import _lib as L
from mordred_b200 import cpu, ssb

pytestmark = pytest.mark.gpu
SEG = 1 << 20


@pytest.fixture(scope="module", autouse=True)
def device():
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    yield
    torch.cuda.synchronize()


def _qb(n, seed):
    s = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(s, seed, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    ssb.build_b(t, ws)
    return s, t, ws


def _qb_probes(s, t, ws):
    return [dict(fkey=t["lo_suppkey"], ht=ws["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_custkey"], ht=ws["ht_c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
                 res_slot=1),
            dict(fkey=t["lo_partkey"], ht=ws["ht_p_b"], num_slots=s.p_len, layout=L.MB_HT_KEY),
            dict(fkey=t["lo_orderdate"], ht=ws["ht_d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                 layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)]


def _expected(s, t, ws, date):
    """(rows, probe outputs) passing the date filter and Query B's four probes: the
    oracle's selection (orc_select) over the same columns and tables, in row order."""
    from oracle import oracle as O
    h = {k: v.cpu().numpy() for k, v in t.items()}
    hw = {k: ws[k].cpu().numpy() for k in ("ht_s", "ht_c", "ht_p_b", "ht_d")}
    probes = [dict(fkey=h["lo_suppkey"], ht=hw["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
              dict(fkey=h["lo_custkey"], ht=hw["ht_c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL),
              dict(fkey=h["lo_partkey"], ht=hw["ht_p_b"], num_slots=s.p_len, layout=L.MB_HT_KEY),
              dict(fkey=h["lo_orderdate"], ht=hw["ht_d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                   layout=L.MB_HT_KEY_VAL)]
    rows, dims, k, st = O.select(len(h["lo_orderdate"]),
                                 filters=[dict(col=h["lo_orderdate"], mode=L.MB_FILTER_BETWEEN, c1=date[0],
                                               c2=date[1])], probes=probes)
    assert st == 0 and k == len(rows)
    return rows, dims


def test_select_offset_list_and_payloads():
    n = 2_000_003
    s, t, ws = _qb(n, 5)
    date = (19940101, 19961231)
    args = ssb.star_args(num_rows=n, filters=[dict(col=t["lo_orderdate"], mode=L.MB_FILTER_BETWEEN, c1=date[0],
                                                   c2=date[1])], probes=_qb_probes(s, t, ws))
    lo = torch.empty(n, dtype=torch.int32, device="cuda")
    dim = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(4)]
    dptr = (C.c_void_p * 4)(*[d.data_ptr() for d in dim])
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("mb_star_select", C.byref(args), None, 0, lo.data_ptr(), dptr, n, total.data_ptr(), ssb._stream())
    k = int(total.item())
    rows, odims = _expected(s, t, ws, date)
    assert k == len(rows) > 0
    order = torch.argsort(lo[:k]).cpu().numpy()
    got_rows = lo[:k].cpu().numpy()[order]
    assert np.array_equal(got_rows, rows)
    for j in range(4):                                                 # payloads: none, nation, none, year
        assert np.array_equal(dim[j][:k].cpu().numpy()[order], odims[j]), j
    assert (dim[0][:k] == 0).all()                                     # KEY layout: no payload
    years = dim[3][:k].cpu().numpy()[order]
    assert years.min() >= 1994 and years.max() <= 1996
    assert L.device_status(0) == 0
    # a list that is too short: every row is counted, the ones past the end are not written
    total.zero_()
    lo.fill_(-1)
    L.call("mb_star_select", C.byref(args), None, 0, lo.data_ptr(), None, 1000, total.data_ptr(), ssb._stream())
    assert int(total.item()) == len(rows)
    assert (lo[:1000] >= 0).all() and (lo[1000:] == -1).all()
    assert L.device_status(0) == L.MB_STATUS_OVERFLOW


def test_split_execution_gpu_select_cpu_aggregate():
    """Rows [0, cut) run the whole query on the GPU; rows [cut, n) are selected on the GPU,
    the offset list goes to the host and the CPU engine aggregates them there. The merged
    result equals the whole query on the GPU, bit for bit."""
    n = 3_000_017
    cut = 1_234_567
    s, t, ws = _qb(n, 9)
    probes = _qb_probes(s, t, ws)
    kw = dict(probes=probes, aggr=[t["lo_revenue"], t["lo_supplycost"]], agg_op=L.MB_AGG_SUB, total_val=175,
              res_layout=L.MB_RES_CRYSTAL4)
    full = torch.zeros(4 * 175, dtype=torch.int32, device="cuda")
    ssb.star_query(ssb.star_args(num_rows=n, res=full, **kw))
    # GPU half
    part = torch.zeros(4 * 175, dtype=torch.int32, device="cuda")
    ssb.star_query(ssb.star_args(num_rows=cut, res=part, **kw))
    # GPU selection of the rest, physical rows = start_offset + row
    tail = {k: v[cut:] for k, v in t.items() if k.startswith("lo_")}
    sel = ssb.star_args(num_rows=n - cut, probes=_qb_probes(s, tail, ws), start_offset=cut)
    lo = torch.empty(n - cut, dtype=torch.int32, device="cuda")
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("mb_star_select", C.byref(sel), None, 0, lo.data_ptr(), None, n - cut, total.data_ptr(), ssb._stream())
    rows = lo[: int(total.item())].cpu().numpy()
    # CPU half over host columns and host copies of the tables, listed rows only
    h = {k: v.cpu().numpy() for k, v in t.items()}
    hw = {k: ws[k].cpu().numpy() for k in ("ht_s", "ht_c", "ht_p_b", "ht_d")}
    hprobes = [dict(fkey=h["lo_suppkey"], ht=hw["ht_s"], num_slots=s.s_len, layout=L.MB_HT_KEY),
               dict(fkey=h["lo_custkey"], ht=hw["ht_c"], num_slots=s.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
                    res_slot=1),
               dict(fkey=h["lo_partkey"], ht=hw["ht_p_b"], num_slots=s.p_len, layout=L.MB_HT_KEY),
               dict(fkey=h["lo_orderdate"], ht=hw["ht_d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                    layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)]
    host_res = part.cpu().numpy().copy()
    assert cpu.star_query(ssb.star_args(num_rows=n, probes=hprobes, aggr=[h["lo_revenue"], h["lo_supplycost"]],
                                        agg_op=L.MB_AGG_SUB, total_val=175, res_layout=L.MB_RES_CRYSTAL4,
                                        res=host_res), rows=rows) == 0
    assert np.array_equal(host_res, full.cpu().numpy())
    assert L.device_status(0) == 0


def _engine(seed=3, nseg=4):
    lo_len = nseg * SEG
    s = ssb.Sizes(lo_len=lo_len, s_len=8_000, c_len=90_000, p_len=150_000)
    fact = ["lo_suppkey", "lo_custkey", "lo_partkey", "lo_orderdate"]
    t = ssb.gen_device(s, seed, fact, ssb.QB_DIMS)
    rng = np.random.default_rng(seed)
    nslots = nseg * len(fact) + 2
    cache = torch.zeros(nslots * SEG, dtype=torch.int32, device="cuda")
    slots = rng.permutation(nslots)[: nseg * len(fact)].reshape(len(fact), nseg)
    col_idx = {}
    for ci, name in enumerate(fact):
        for sg in range(nseg):
            cache[int(slots[ci, sg]) * SEG: (int(slots[ci, sg]) + 1) * SEG] = t[name][sg * SEG:(sg + 1) * SEG]
        col_idx[name] = torch.from_numpy(slots[ci].astype(np.int32)).cuda()
    hts = {}
    for name, key, val, flt, mode, c1, c2, nsl, kmin in [
            ("s", "s_suppkey", "s_region", "s_region", 1, 1, 1, s.s_len, 0),
            ("c", "c_custkey", "c_nation", "c_region", 1, 1, 1, s.c_len, 0),
            ("d", "d_datekey", "d_year", None, 0, 0, 0, ssb.DATE_SLOTS, ssb.DATE_MIN)]:
        ht = torch.zeros(2 * nsl, dtype=torch.int32, device="cuda")
        f = L.MbFilterArgsGPU(ssb._p(t[flt]) if flt else None, None, c1, c2, 0, 0, mode, 0)
        b = L.MbBuildArgsGPU(ssb._p(t[key]), ssb._p(t[val]), nsl, kmin, 0)
        L.call("mb_build_GPU2", None, C.byref(f), C.byref(b), t[key].numel(), ssb._p(ht), 0, None, ssb._stream())
        hts[name] = (ht, nsl, kmin)
    return s, t, cache, col_idx, hts


def test_engine_compaction_gpu2_then_gpu3():
    s, t, cache, col_idx, hts = _engine()
    h = {k: v.cpu().numpy().astype(np.int64) for k, v in t.items()}
    segs = torch.tensor([2, 0, 3], dtype=torch.int16, device="cuda")
    nt = 3 * SEG
    f = L.MbFilterArgsGPU(ssb._p(col_idx["lo_orderdate"]), None, 19930101, 19951231, 0, 0, L.MB_FILTER_BETWEEN, 0)
    p = L.MbProbeArgsGPU()
    p.key_idx1, p.ht1, p.dim_len1 = ssb._p(col_idx["lo_suppkey"]), ssb._p(hts["s"][0]), hts["s"][1]
    buf = [torch.full((nt,), -7, dtype=torch.int32, device="cuda") for _ in range(5)]
    out = L.MbOffsetGPU(*[b.data_ptr() for b in buf])
    out.dim_off2 = out.dim_off3 = out.dim_off4 = None
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("mb_filter_probe_GPU2", ssb._p(cache), C.byref(f), C.byref(p), C.byref(out), nt, total.data_ptr(), 0,
           segs.data_ptr(), ssb._stream())
    k = int(total.item())
    phys = np.concatenate([np.arange(sg * SEG, (sg + 1) * SEG) for sg in (2, 0, 3)])
    od = h["lo_orderdate"][phys]
    hs = hts["s"][0].cpu().numpy()
    srow = hs[2 * (h["lo_suppkey"][phys] % s.s_len) + 1]
    ok = (od >= 19930101) & (od <= 19951231) & (srow != 0)
    exp_rows = np.sort(phys[ok])
    assert k == len(exp_rows)
    lo = buf[0][:k].cpu().numpy()
    order = np.argsort(lo)
    assert np.array_equal(lo[order], exp_rows)
    exp_dim1 = (hs[2 * (h["lo_suppkey"] % s.s_len) + 1] - 1)[exp_rows]
    assert np.array_equal(buf[1][:k].cpu().numpy()[order], exp_dim1)     # supplier row offsets
    # second stage over the list: probe customer and date, pass the supplier offsets through
    p2 = L.MbProbeArgsGPU()
    p2.key_idx2, p2.ht2, p2.dim_len2 = ssb._p(col_idx["lo_custkey"]), ssb._p(hts["c"][0]), hts["c"][1]
    p2.key_idx4, p2.ht4, p2.dim_len4, p2.min_key4 = (ssb._p(col_idx["lo_orderdate"]), ssb._p(hts["d"][0]),
                                                     hts["d"][1], hts["d"][2])
    buf2 = [torch.full((k,), -7, dtype=torch.int32, device="cuda") for _ in range(5)]
    out2 = L.MbOffsetGPU(*[b.data_ptr() for b in buf2])
    out2.dim_off3 = None
    in_off = L.MbOffsetGPU(buf[0].data_ptr(), buf[1].data_ptr(), None, None, None)
    total2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.call("mb_probe_GPU3", ssb._p(cache), C.byref(in_off), C.byref(p2), C.byref(out2), k, total2.data_ptr(),
           ssb._stream())
    k2 = int(total2.item())
    hc = hts["c"][0].cpu().numpy()
    crow = hc[2 * (h["lo_custkey"][exp_rows] % s.c_len) + 1]
    keep = crow != 0
    assert k2 == int(keep.sum()) > 0
    lo2 = buf2[0][:k2].cpu().numpy()
    o2 = np.argsort(lo2)
    assert np.array_equal(lo2[o2], exp_rows[keep])
    assert np.array_equal(buf2[1][:k2].cpu().numpy()[o2], exp_dim1[keep])       # passed through
    assert np.array_equal(buf2[2][:k2].cpu().numpy()[o2], crow[keep] - 1)        # customer row offsets
    drow = hts["d"][0].cpu().numpy()[2 * (h["lo_orderdate"][exp_rows[keep]] - ssb.DATE_MIN) + 1] - 1
    assert np.array_equal(buf2[4][:k2].cpu().numpy()[o2], drow)                  # date row offsets
    assert L.device_status(0) == 0
