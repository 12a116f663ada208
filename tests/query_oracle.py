"""Expected results of the workload's query forms (filter-aggregate, Query A, Query B with
range predicates) from the CPU oracle: filtered builds with orc_build, then orc_star over
the fact rows — the reference's way of running one query, restated on the host. Used by
the tests to pin batched, segmented and served results to the oracle rather than to
another CUDA run."""
import numpy as np

from mordred_b200 import ssb
from oracle import oracle as O


def _table(h, flt, lo, hi, key, val, slots, kmin, layout):
    ht = np.zeros(2 * slots if layout else slots, np.int32)
    st = O.build_ht(h[flt] if flt else None, 1, lo, hi, h[key], h[val] if val else None, ht, slots, kmin, layout)
    assert st == 0
    return ht


def expected(h: dict, sizes: ssb.Sizes, q, n_rows: int | None = None, rows=None, segment_group=None,
             segment_size: int = 0) -> np.ndarray:
    """The result array of query q (a batch.Query) over the host columns h, laid out as
    q.result_buffer(): int64[1] for the filter-aggregate, int32[4*G] {key0, key1, u64 sum}
    otherwise. n_rows defaults to the fact table's length."""
    n = len(h["lo_orderdate"]) if n_rows is None else n_rows
    seg = dict(rows=rows, segment_group=segment_group, segment_size=segment_size)
    date = dict(col=h["lo_orderdate"], mode=1, c1=q.date[0], c2=q.date[1])
    if q.template == "agg":
        res = np.zeros(1, np.uint64)
        st = O.star(n, filters=[date, dict(col=h["lo_discount"], mode=1, c1=q.discount[0], c2=q.discount[1]),
                                dict(col=h["lo_quantity"], mode=1, c1=q.quantity[0], c2=q.quantity[1])],
                    aggr=[h["lo_extendedprice"], h["lo_discount"]], agg_op=2, res_layout=0, res=res, **seg)
        assert st == 0
        return res.view(np.int64)
    ht_s = _table(h, "s_region", *q.s_region, "s_suppkey", None, sizes.s_len, 0, 0)
    ht_d = _table(h, None, 0, 0, "d_datekey", "d_year", ssb.DATE_SLOTS, ssb.DATE_MIN, 1)
    d_probe = dict(fkey=h["lo_orderdate"], ht=ht_d, num_slots=ssb.DATE_SLOTS, key_min=ssb.DATE_MIN, layout=1,
                   min_val=1992, unique_val=1, res_slot=0)
    s_probe = dict(fkey=h["lo_suppkey"], ht=ht_s, num_slots=sizes.s_len, layout=0)
    if q.template == "qa":
        ht_p = _table(h, "p_category", *q.category, "p_partkey", "p_brand1", sizes.p_len, 0, 1)
        res = np.zeros(4 * ssb.QA_GROUPS, np.int32)
        st = O.star(n, filters=[date],
                    probes=[s_probe, dict(fkey=h["lo_partkey"], ht=ht_p, num_slots=sizes.p_len, layout=1,
                                          unique_val=7, res_slot=1), d_probe],
                    aggr=[h["lo_revenue"]], agg_op=0, total_val=ssb.QA_GROUPS, res_layout=2, res=res, **seg)
    else:
        ht_c = _table(h, "c_region", *q.c_region, "c_custkey", "c_nation", sizes.c_len, 0, 1)
        ht_p = _table(h, "p_mfgr", *q.mfgr, "p_partkey", None, sizes.p_len, 0, 0)
        res = np.zeros(4 * ssb.QB_GROUPS, np.int32)
        st = O.star(n, filters=[date],
                    probes=[s_probe, dict(fkey=h["lo_custkey"], ht=ht_c, num_slots=sizes.c_len, layout=1,
                                          unique_val=7, res_slot=1),
                            dict(fkey=h["lo_partkey"], ht=ht_p, num_slots=sizes.p_len, layout=0), d_probe],
                    aggr=[h["lo_revenue"], h["lo_supplycost"]], agg_op=1, total_val=ssb.QB_GROUPS, res_layout=2,
                    res=res, **seg)
    assert st == 0
    return res
