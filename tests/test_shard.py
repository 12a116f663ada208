"""The multi-GPU path's host logic on CPU ranks (gloo, world size 2): each rank takes its
row shard of the one seeded table, answers Query B on it (the CPU engine stands in for
its GPU), and one all-reduce of the dense group sums gives the whole table's answer."""
import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from mordred_b200 import _lib as L
from mordred_b200 import cpu, shard, ssb

N = 150_001  # rows per rank
SIZES = ssb.Sizes(lo_len=N, s_len=2_000, c_len=30_000, p_len=20_000)


def _qb(t: dict, d: dict, n: int) -> np.ndarray:
    hts = {}
    for name, flt, mode, c1, c2, key, val, slots, kmin, layout in [
            ("s", "s_region", L.MB_FILTER_EQ, 1, 0, "s_suppkey", None, SIZES.s_len, 0, L.MB_HT_KEY),
            ("c", "c_region", L.MB_FILTER_EQ, 1, 0, "c_custkey", "c_nation", SIZES.c_len, 0, L.MB_HT_KEY_VAL),
            ("p", "p_mfgr", L.MB_FILTER_EQ_OR_EQ, 0, 1, "p_partkey", None, SIZES.p_len, 0, L.MB_HT_KEY),
            ("d", None, 0, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN, L.MB_HT_KEY_VAL)]:
        ht = np.zeros(slots if layout == L.MB_HT_KEY else 2 * slots, np.int32)
        cpu.build_pht(d[flt] if flt else None, mode, c1, c2, d[key], d[val] if val else None, ht, slots, kmin, layout)
        hts[name] = ht
    probes = [dict(fkey=t["lo_suppkey"], ht=hts["s"], num_slots=SIZES.s_len, layout=L.MB_HT_KEY),
              dict(fkey=t["lo_custkey"], ht=hts["c"], num_slots=SIZES.c_len, layout=L.MB_HT_KEY_VAL, unique_val=7,
                   res_slot=1),
              dict(fkey=t["lo_partkey"], ht=hts["p"], num_slots=SIZES.p_len, layout=L.MB_HT_KEY),
              dict(fkey=t["lo_orderdate"], ht=hts["d"], num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN,
                   layout=L.MB_HT_KEY_VAL, min_val=1992, unique_val=1, res_slot=0)]
    res = np.zeros(4 * ssb.QB_GROUPS, np.int32)
    cpu.star_query(ssb.star_args(num_rows=n, probes=probes, aggr=[t["lo_revenue"], t["lo_supplycost"]],
                                 agg_op=L.MB_AGG_SUB, total_val=ssb.QB_GROUPS, res_layout=L.MB_RES_CRYSTAL4,
                                 res=res), nthreads=2)
    return res


def _rank(rank: int, world: int, port: int, out: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = {k: v.numpy() for k, v in shard.gen_shard(SIZES, 7, ssb.QB_FACT, rank, N, device="cpu").items()}
        d = ssb.gen_host(SIZES, 7, [], ssb.QB_DIMS)
        res = torch.from_numpy(_qb(t, d, N))
        dense = torch.zeros(ssb.QB_GROUPS, dtype=torch.int64)
        shard.allreduce_sums([shard.crystal4_sums(res)], dense)
        if rank == 0:
            np.save(out, dense.numpy())
    finally:
        dist.destroy_process_group()


def test_row_shards_and_allreduce_equal_the_whole_table(tmp_path):
    out = str(tmp_path / "dense.npy")
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    whole = ssb.Sizes(lo_len=2 * N, s_len=SIZES.s_len, c_len=SIZES.c_len, p_len=SIZES.p_len)
    t = ssb.gen_host(whole, 7, ssb.QB_FACT, ssb.QB_DIMS)
    exp = shard.crystal4_sums(torch.from_numpy(_qb(t, t, 2 * N))).numpy()
    got = np.load(out)
    assert np.array_equal(got, exp) and (exp != 0).any()
