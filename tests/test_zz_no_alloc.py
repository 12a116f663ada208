"""GPU test of mb_q41_probe_noalloc, the Query B probe for callers that cannot allocate
device memory (an executor whose device buffers all come from its own arena, or a
thread that must not synchronise the device through cudaMalloc).

The entry point is called through the C ABI twice in a row and each result is compared
bit for bit with mb_q41_probe's on the same inputs (integer sums: the tolerance is zero).
The file name sorts last so that, in a run stopping at the first failure, every other
test has run before it; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mordred_b200 import _lib as L
from mordred_b200 import ssb

pytestmark = pytest.mark.gpu


def _probe_args(t, ws, s):
    return [ssb._p(t[k]) for k in ("lo_orderdate", "lo_partkey", "lo_custkey", "lo_suppkey", "lo_revenue",
                                   "lo_supplycost")] + \
           [s.lo_len, ssb._p(ws["ht_p_b"]), s.p_len, ssb._p(ws["ht_s"]), s.s_len, ssb._p(ws["ht_c"]), s.c_len,
            ssb._p(ws["ht_d"]), ssb.DATE_SLOTS]


def test_noalloc_probe_matches_allocating_probe_twice():
    torch.cuda.set_device(0)
    s = ssb.Sizes(lo_len=3_000_017, s_len=40_000, c_len=600_000, p_len=1_000_000)
    t = ssb.gen_device(s, 4242, ssb.QB_FACT, ssb.QB_DIMS)
    ws = ssb.StarWorkspace(s)
    ssb.build_b(t, ws)          # hash tables (and a zeroed res_b) for both probes
    torch.cuda.synchronize()
    lib = L.lib()
    stream = ssb._stream()
    status = torch.full((1,), 0x7fffffff, dtype=torch.int32, device="cuda")
    for call in range(2):
        res_na = torch.zeros(4 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
        rc = lib.mb_q41_probe_noalloc(*_probe_args(t, ws, s), ssb._p(res_na), ssb._p(status), stream)
        assert rc == 0, lib.mb_error_string(rc).decode()
        res_ref = torch.zeros(4 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
        rc = lib.mb_q41_probe(*_probe_args(t, ws, s), ssb._p(res_ref), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(status.item()) == 0, f"call {call}: status {int(status.item()):#x}"
        a, b = res_na.cpu().numpy(), res_ref.cpu().numpy()
        assert np.array_equal(a, b), f"call {call} differs"
        assert len(ssb.crystal4_groups(a)) > 0


def test_noalloc_rejects_supplier_table_beyond_scratch():
    lib = L.lib()
    big = 262_144 + 1
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = ssb._p(dummy)
    rc = lib.mb_q41_probe_noalloc(p, p, p, p, p, p, 4, p, 4, p, big, p, 4, p, 4, p, None, ssb._stream())
    assert rc == 6  # MB_ERR_SIZE
    assert "size" in lib.mb_error_string(rc).decode()
