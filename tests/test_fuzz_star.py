"""Randomised star queries against the oracle, bit for bit and with equal status bits.

Each case draws 0-3 fact filters of every mode (empty BETWEEN ranges included), 0-4
probes over tables of all three layouts (4 B key slots, {key, val} and {val, row + 1}
8-byte slots) with sizes on both sides of the shared-memory bitmap limits, key_min
offsets, fills from empty to full and some keys below key_min (a probe-range status),
group multipliers and minima that can push rows outside [0, total_val) (a group-range
status), every aggregate and every result layout, a selection count after a random
filter, caller-supplied presence bitmaps, and a random launch shape. The CUDA kernel
(`mb_star_query`, gpu; direct columns and segment-cache addressing) and the library's
CPU operator (`mb_cpu_star_query`) must both reproduce the oracle's result array and
status bits.
"""
import numpy as np
import pytest
import torch

from mordred_b200 import _lib as L
from mordred_b200 import cpu, ssb
from oracle import oracle as O


def make_case(seed: int, n: int | None = None) -> dict:
    rng = np.random.default_rng(seed)
    drawn = int(rng.choice([0, 1, 33, 2048, 4099, 65_537, 250_001, 1_000_003]))
    n = drawn if n is None else n

    def fact_col(lo, hi):
        return rng.integers(lo, hi, n, dtype=np.int64).astype(np.int32)

    filters = []
    for _ in range(int(rng.integers(0, L.MB_MAX_FILTERS + 1))):
        mode = int(rng.integers(0, 3))
        c1, c2 = int(rng.integers(0, 10)), int(rng.integers(0, 10))
        if mode == L.MB_FILTER_BETWEEN and rng.random() < 0.85:
            c1, c2 = min(c1, c2), max(c1, c2)
        filters.append(dict(col=fact_col(0, 10), mode=mode, c1=c1, c2=c2))

    res_layout = int(rng.choice([L.MB_RES_SCALAR, L.MB_RES_ENGINE6, L.MB_RES_CRYSTAL4, L.MB_RES_DENSE]))
    max_res_slot = {L.MB_RES_ENGINE6: 3, L.MB_RES_CRYSTAL4: 1}.get(res_layout, -1)
    nprobes = int(rng.integers(0 if filters else 1, L.MB_MAX_PROBES + 1))
    # With key-writing layouts, a "structured" case makes the group index a mixed-radix
    # number of the key-writing probes' payloads, so every group has one key tuple and
    # the written keys are defined; otherwise groups may mix key tuples (whose keys the
    # reference leaves to the last writer) and only the sums are compared.
    structured = max_res_slot >= 0 and rng.random() < 0.6
    key_slots = list(rng.permutation(max_res_slot + 1)) if max_res_slot >= 0 else []
    radix = 1
    probes = []
    for _ in range(nprobes):
        slots = int(rng.choice([64, 1000, 40_000, 65_536, 70_001, 300_000]))
        layout = int(rng.integers(0, 3))
        kmin = int(rng.choice([0, 1, -5, 19920101]))
        present = rng.random(slots) < float(rng.choice([0.0, 0.05, 0.5, 0.9, 1.0], p=[0.05, 0.15, 0.3, 0.3, 0.2]))
        nonzero = rng.integers(1, 2**31 - 1, slots).astype(np.int32)
        min_val, unique_val = int(rng.integers(-3, 3)), int(rng.integers(0, 8))
        res_slot = int(rng.integers(-1, max_res_slot + 1)) if max_res_slot >= 0 else -1
        payload = rng.integers(-3, 40, slots).astype(np.int32)
        if structured:
            res_slot = int(key_slots.pop()) if key_slots and rng.random() < 0.8 else -1
            if res_slot >= 0:
                r = int(rng.integers(1, 12))
                payload = rng.integers(min_val, min_val + r, slots).astype(np.int32)
                unique_val, radix = radix, radix * r
            else:
                unique_val = 0
        if layout == L.MB_HT_KEY:
            ht = np.where(present, nonzero, 0).astype(np.int32)
        else:
            ht = np.zeros(2 * slots, np.int32)
            lo, hi = (nonzero, payload) if layout == L.MB_HT_KEY_VAL else (payload, nonzero)
            ht[0::2] = np.where(present, lo, 0)
            ht[1::2] = np.where(present, hi, 0)
        below = int(rng.choice([0, 0, 0, 3]))  # keys down to key_min - 3: probe-range status
        fkey = (kmin + rng.integers(-below, slots + slots // 3, n)).astype(np.int32)
        q = dict(fkey=fkey, ht=ht, num_slots=slots, key_min=kmin, layout=layout, min_val=min_val,
                 unique_val=unique_val, res_slot=res_slot)
        if rng.random() < 0.3:
            # bit j of word w: slot 32 w + j is occupied
            occ = ht != 0 if layout == L.MB_HT_KEY else (ht[0::2] != 0) | (ht[1::2] != 0)
            idx = np.nonzero(occ)[0]
            words = np.zeros((slots + 31) // 32, np.uint32)
            np.bitwise_or.at(words, idx >> 5, (np.uint32(1) << (idx & 31).astype(np.uint32)))
            q["presence"] = words
        probes.append(q)

    ops = [L.MB_AGG_SUM, L.MB_AGG_SUB, L.MB_AGG_MUL]
    if probes and probes[0]["layout"] != L.MB_HT_KEY:
        ops.append(L.MB_AGG_MUL_PAYLOAD)
    agg_op = int(rng.choice(ops))
    aggr = [fact_col(-10**6, 10**7), fact_col(-10**5, 10**6)]
    total_val = 1 if res_layout == L.MB_RES_SCALAR else int(rng.choice([1, 7, 175, 1000, 7000, 9000]))
    if structured:
        total_val = radix * int(rng.choice([1, 2]))
    count_after = int(rng.integers(-1, len(filters) + 1)) if rng.random() < 0.5 else None
    launch = dict(threads=int(rng.choice([0, 128, 256, 512])), items_per_thread=int(rng.choice([0, 4, 8, 16])),
                  stages=int(rng.choice([0, 2, 3])), grid=int(rng.choice([0, 0, 1, 7])),
                  group_mode=int(rng.choice([0, 2] + ([1] if total_val <= 8192 else []))))
    return dict(n=n, filters=filters, probes=probes, aggr=aggr if agg_op != L.MB_AGG_SUM else aggr[:1],
                agg_op=agg_op, total_val=total_val, group_bias=int(rng.integers(0, 100)), res_layout=res_layout,
                count_after=count_after, launch=launch, keys_defined=max_res_slot < 0 or structured)


def comparable(case, res):
    """The result fields the reference defines: all of them, or only the sums where a
    group may mix key tuples."""
    if case["keys_defined"]:
        return res
    w = 6 if case["res_layout"] == L.MB_RES_ENGINE6 else 4
    return res.reshape(-1, w)[:, w - 2:].copy()


def result_array(case):
    tv, rl = case["total_val"], case["res_layout"]
    if rl == L.MB_RES_SCALAR:
        return np.zeros(1, np.uint64)
    if rl == L.MB_RES_DENSE:
        return np.zeros(tv, np.uint64)
    return np.zeros((6 if rl == L.MB_RES_ENGINE6 else 4) * tv, np.int32)


def oracle_run(case, rows=None, **segments):
    res = result_array(case)
    cnt = np.zeros(1, np.uint64)
    st = O.star(case["n"] if rows is None else rows, filters=case["filters"], probes=case["probes"],
                aggr=case["aggr"], agg_op=case["agg_op"], total_val=case["total_val"], group_bias=case["group_bias"],
                res_layout=case["res_layout"], res=res, count=cnt if case["count_after"] is not None else None,
                count_after=case["count_after"] if case["count_after"] is not None else -1, **segments)
    return res, int(cnt[0]), st


def args_for(case, conv, res, cnt, launch, rows=None):
    """MbStarArgs with every array passed through `conv` (host numpy or device tensor)."""
    filters = [dict(f, col=conv(f["col"])) for f in case["filters"]]
    probes = []
    for q in case["probes"]:
        d = dict(q, fkey=conv(q["fkey"]), ht=conv(q["ht"]))
        if "presence" in q:
            d["presence"] = conv(q["presence"].view(np.int32))
        probes.append(d)
    kw = dict(launch)
    if case["count_after"] is not None:
        kw.update(count=cnt, count_after=case["count_after"])
    return ssb.star_args(num_rows=case["n"] if rows is None else rows, filters=filters, probes=probes,
                         aggr=[conv(a) for a in case["aggr"]], agg_op=case["agg_op"], total_val=case["total_val"], group_bias=case["group_bias"],
                         res_layout=case["res_layout"], res=res, **kw)


@pytest.mark.parametrize("seed", range(40))
def test_cpu_operator_matches_oracle(seed):
    case = make_case(1000 + seed)
    exp, ecnt, est = oracle_run(case)
    res = result_array(case)
    cnt = np.zeros(1, np.uint64)
    st = cpu.star_query(args_for(case, lambda a: a, res, cnt, {}))
    assert st == est
    assert np.array_equal(comparable(case, res), comparable(case, exp))
    if case["count_after"] is not None:
        assert int(cnt[0]) == ecnt


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(120))
def test_cuda_kernel_matches_oracle(seed):
    case = make_case(5000 + seed)
    exp, ecnt, est = oracle_run(case)
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    keep = []

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        keep.append(t)
        return t

    for launch in (case["launch"], {}):
        res = dev(result_array(case))
        cnt = dev(np.zeros(1, np.uint64))
        try:
            ssb.star_query(args_for(case, dev, res, cnt, launch))
        except L.MbError as e:
            # a drawn launch shape whose stages cannot fit next to this case's columns
            assert e.code == L.MB_ERR_SIZE and launch, e
            continue
        torch.cuda.synchronize()
        assert L.device_status(0, clear=True) == est, launch
        assert np.array_equal(comparable(case, res.cpu().numpy()), comparable(case, exp)), launch
        if case["count_after"] is not None:
            assert int(cnt.cpu().numpy()[0]) == ecnt, launch


def _fact_arrays(case):
    cols = [f["col"] for f in case["filters"]] + [q["fkey"] for q in case["probes"]] + list(case["aggr"])
    return list({id(a): a for a in cols}.values())


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(60))
def test_cuda_kernel_segment_cache_matches_oracle(seed):
    """The same random queries over a segment cache: every fact column's segments sit at
    shuffled slots of one cache array (the engine's gpuCache), columns are per-segment
    slot indices, and the call's rows are either a list of segments (a permutation of a
    subset, the last one cut short) or a run from a segment-aligned start offset."""
    rng = np.random.default_rng(9000 + seed)
    seg = int(rng.choice([1 << 14, 1 << 16]))
    nphys = int(rng.integers(1, 7))
    case = make_case(9000 + seed, n=nphys * seg)
    if rng.random() < 0.5:
        k = int(rng.integers(1, nphys + 1))
        seg_list = rng.permutation(nphys)[:k].astype(np.int16)
        start, rows = 0, k * seg - int(rng.integers(0, seg))
    else:
        seg_list = None
        j = int(rng.integers(0, nphys))
        start, rows = j * seg, int(rng.integers(0, (nphys - j) * seg + 1))
    exp, ecnt, est = oracle_run(case, rows, segment_group=seg_list, start_offset=start, segment_size=seg)

    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    keep = []

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        keep.append(t)
        return t

    facts = _fact_arrays(case)
    nslots = len(facts) * nphys + 2
    perm = rng.permutation(nslots)
    cache = np.zeros(nslots * seg, np.int32)
    col_idx = {}
    for ci, arr in enumerate(facts):
        slots = perm[ci * nphys:(ci + 1) * nphys]
        for sg in range(nphys):
            cache[slots[sg] * seg:(slots[sg] + 1) * seg] = arr[sg * seg:(sg + 1) * seg]
        col_idx[id(arr)] = dev(slots.astype(np.int32))
    cache_dev = dev(cache)
    seg_dev = dev(seg_list) if seg_list is not None else None

    def conv(a):
        return col_idx[id(a)] if id(a) in col_idx else dev(a)

    for launch in (case["launch"], {}):
        res = dev(result_array(case))
        cnt = dev(np.zeros(1, np.uint64))
        kw = dict(launch, gpu_cache=cache_dev, segment_group=seg_dev, start_offset=start, segment_size=seg)
        try:
            ssb.star_query(args_for(case, conv, res, cnt, kw, rows=rows))
        except L.MbError as e:
            assert e.code == L.MB_ERR_SIZE and launch, e
            continue
        torch.cuda.synchronize()
        assert L.device_status(0, clear=True) == est, launch
        assert np.array_equal(comparable(case, res.cpu().numpy()), comparable(case, exp)), launch
        if case["count_after"] is not None:
            assert int(cnt.cpu().numpy()[0]) == ecnt, launch
