"""The Crystal block-primitive API (include/crystal_b200.cuh).

* CPU: the header compiles at the language level Crystal code is written for (C++14),
  and the reference's own Crystal programs compile against it (oracle/_ref, built by
  oracle/Makefile where the reference tree is present).
* GPU: star-query programs written against the API (tests/crystal/crystal_programs.cu)
  and the reference's own programs src/ssb/q11.cu, q21.cu, q41.cu compiled unmodified
  against the header (their kernels, launched as their runQuery launches them) compute
  the oracle's answers bit for bit.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from mordred_b200 import ssb
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PROGRAMS = os.path.join(HERE, "crystal", "libcrystal_programs.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libcrystal_ref_q{}.so")


def test_header_compiles_as_cxx14():
    r = subprocess.run(["make", "-s", "-C", os.path.join(HERE, "crystal"), "check14"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def test_reference_programs_built_against_the_header():
    import __graft_entry__
    if not __graft_entry__.reference_tree() and not all(os.path.exists(REF_LIB.format(q)) for q in (11, 21, 41)):
        pytest.skip("no reference tree to build from and no prebuilt reference programs")
    for q in (11, 21, 41):
        assert os.path.exists(REF_LIB.format(q)), f"oracle/_ref/libcrystal_ref_q{q}.so was not built"


def _programs():
    if not os.path.exists(PROGRAMS):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "crystal")], check=True)
    lib = C.CDLL(PROGRAMS)
    for name in ("cp_filter_aggregate", "cp_build", "cp_probe_brand_year", "cp_probe_nation_year"):
        getattr(lib, name).restype = C.c_int
    return lib


def _tables(sizes, seed, d_len):
    import torch
    s = ssb.Sizes(lo_len=sizes[0], s_len=sizes[1], c_len=sizes[2], p_len=sizes[3], d_len=d_len)
    cols = ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"]
    dims = sorted(set(ssb.QA_DIMS + ssb.QB_DIMS))
    h = ssb.gen_host(s, seed, cols, dims)
    d = {k: torch.from_numpy(v).cuda() for k, v in h.items()}
    return s, h, d


P = lambda t: C.c_void_p(t.data_ptr())


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 511, 512, 513, 1_000_003, 6_000_000])
def test_crystal_programs_filter_aggregate(n):
    import torch
    lib = _programs()
    s, h, d = _tables((n, 100, 300, 200), 31 + n, 2557)
    rev = torch.zeros(1, dtype=torch.int64, device="cuda")
    assert lib.cp_filter_aggregate(P(d["lo_orderdate"]), P(d["lo_discount"]), P(d["lo_quantity"]),
                                   P(d["lo_extendedprice"]), n, P(rev)) == 0
    assert int(rev.item()) % 2**64 == O.q11(h)


@pytest.mark.gpu
@pytest.mark.parametrize("sizes", [(1000, 100, 300, 200), (3_000_017, 40_000, 600_000, 1_000_000)])
def test_crystal_programs_query_a_and_b(sizes):
    import torch
    lib = _programs()
    s, h, d = _tables(sizes, 5, 2557)
    z = lambda n: torch.zeros(n, dtype=torch.int32, device="cuda")
    ht_s, ht_p, ht_d = z(s.s_len), z(2 * s.p_len), z(2 * ssb.DATE_SLOTS)
    # Query A: supplier region 1, part category 1, the whole date table
    assert lib.cp_build(P(d["s_region"]), 1, -1, P(d["s_suppkey"]), None, s.s_len, P(ht_s), s.s_len, 0) == 0
    assert lib.cp_build(P(d["p_category"]), 1, -1, P(d["p_partkey"]), P(d["p_brand1"]), s.p_len, P(ht_p), s.p_len,
                        0) == 0
    assert lib.cp_build(None, 0, -1, P(d["d_datekey"]), P(d["d_year"]), s.d_len, P(ht_d), ssb.DATE_SLOTS,
                        19920101) == 0
    res = z(4 * ssb.QA_GROUPS)
    assert lib.cp_probe_brand_year(P(d["lo_orderdate"]), P(d["lo_partkey"]), P(d["lo_suppkey"]), P(d["lo_revenue"]),
                                   s.lo_len, P(ht_s), s.s_len, P(ht_p), s.p_len, P(ht_d), ssb.DATE_SLOTS,
                                   P(res)) == 0
    exp, st = O.q21(h, ssb.DATE_SLOTS)
    assert st == 0
    assert ssb.crystal4_groups(res.cpu().numpy()) == O.q21_groups(exp)
    # Query B: customer and supplier region 1, mfgr 0 or 1
    ht_s2, ht_c, ht_pk = z(s.s_len), z(2 * s.c_len), z(s.p_len)
    assert lib.cp_build(P(d["s_region"]), 1, -1, P(d["s_suppkey"]), None, s.s_len, P(ht_s2), s.s_len, 0) == 0
    assert lib.cp_build(P(d["c_region"]), 1, -1, P(d["c_custkey"]), P(d["c_nation"]), s.c_len, P(ht_c), s.c_len,
                        0) == 0
    assert lib.cp_build(P(d["p_mfgr"]), 0, 1, P(d["p_partkey"]), None, s.p_len, P(ht_pk), s.p_len, 0) == 0
    res_b = z(4 * ssb.QB_GROUPS)
    assert lib.cp_probe_nation_year(P(d["lo_orderdate"]), P(d["lo_partkey"]), P(d["lo_custkey"]),
                                    P(d["lo_suppkey"]), P(d["lo_revenue"]), P(d["lo_supplycost"]), s.lo_len,
                                    P(ht_pk), s.p_len, P(ht_s2), s.s_len, P(ht_c), s.c_len, P(ht_d),
                                    ssb.DATE_SLOTS, P(res_b)) == 0
    exp_b, st = O.q41(h, ssb.DATE_SLOTS)
    assert st == 0
    assert np.array_equal(res_b.cpu().numpy(), exp_b)


def _ref_lib(q):
    path = REF_LIB.format(q)
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, ROOT)} not built (the reference tree was absent at build time)")
    lib = C.CDLL(path)
    getattr(lib, f"crystal_ref_q{q}").restype = C.c_int
    return lib


@pytest.mark.gpu
@pytest.mark.parametrize("n", [513, 2_000_003])
def test_reference_q11_program_on_the_header(n):
    """src/ssb/q11.cu's QueryKernel (its BlockLoad / BlockPred* / BlockSum<long long> and
    BlockSum<int> calls) run on this header: revenue and the row count it keeps."""
    import torch
    lib = _ref_lib(11)
    s, h, d = _tables((n, 100, 300, 200), 77, 2556)
    rev = torch.zeros(1, dtype=torch.int64, device="cuda")
    total = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.crystal_ref_q11(P(d["lo_orderdate"]), P(d["lo_discount"]), P(d["lo_quantity"]),
                               P(d["lo_extendedprice"]), n, P(rev), P(total)) == 0
    assert int(rev.item()) % 2**64 == O.q11(h)
    # the count the kernel keeps: rows passing its quantity and discount predicates
    disc, qty = h["lo_discount"], h["lo_quantity"]
    assert int(total.item()) == int(((qty < 25) & (disc >= 1) & (disc <= 3)).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("sizes", [(1000, 100, 300, 200), (3_000_017, 40_000, 600_000, 1_000_000)])
def test_reference_q21_q41_programs_on_the_header(sizes):
    """src/ssb/q21.cu and q41.cu — builds and probe — run on this header over the
    reference's 2,556-row date table with its 61,130 date slots, against the oracle's
    restatement of the reference CPU engine."""
    import torch
    s, h, d = _tables(sizes, 19, 2556)
    z = lambda n: torch.zeros(n, dtype=torch.int32, device="cuda")
    dv = ssb.REFERENCE_DATE_SLOTS
    lib = _ref_lib(21)
    res = z(4 * ssb.QA_GROUPS)
    assert lib.crystal_ref_q21(P(d["lo_orderdate"]), P(d["lo_partkey"]), P(d["lo_suppkey"]), P(d["lo_revenue"]),
                               s.lo_len, P(d["p_partkey"]), P(d["p_brand1"]), P(d["p_category"]), s.p_len,
                               P(d["d_datekey"]), P(d["d_year"]), s.d_len, P(d["s_suppkey"]), P(d["s_region"]),
                               s.s_len, dv, P(z(2 * s.s_len)), P(z(2 * s.p_len)), P(z(2 * dv)), P(res)) == 0
    exp, st = O.q21(h, dv)
    assert st == 0
    assert ssb.crystal4_groups(res.cpu().numpy()) == O.q21_groups(exp)
    lib = _ref_lib(41)
    res_b = z(4 * ssb.QB_GROUPS)
    assert lib.crystal_ref_q41(P(d["lo_orderdate"]), P(d["lo_custkey"]), P(d["lo_partkey"]), P(d["lo_suppkey"]),
                               P(d["lo_revenue"]), P(d["lo_supplycost"]), s.lo_len, P(d["d_datekey"]),
                               P(d["d_year"]), s.d_len, P(d["p_partkey"]), P(d["p_mfgr"]), s.p_len,
                               P(d["s_suppkey"]), P(d["s_region"]), s.s_len, P(d["c_custkey"]), P(d["c_region"]),
                               P(d["c_nation"]), s.c_len, dv, P(z(2 * s.s_len)), P(z(2 * s.c_len)),
                               P(z(2 * s.p_len)), P(z(2 * dv)), P(res_b)) == 0
    exp_b, st = O.q41(h, dv)
    assert st == 0
    assert np.array_equal(res_b.cpu().numpy(), exp_b)
