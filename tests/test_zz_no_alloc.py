"""GPU test of mb_q41_probe_noalloc, the Query B probe for callers that cannot allocate
device memory (an executor whose device buffers all come from its own arena, or a
thread that must not synchronise the device through cudaMalloc).

The entry point is called through the C ABI twice in a row and each result is compared
bit for bit with mb_q41_probe's on the same inputs (integer sums: the tolerance is zero)
and with the CPU oracle's Query B. A second test runs it in a fresh process where nothing
else of the library has run — inputs generated on the host, hash tables built by the
oracle and copied in — and checks that the library's allocating per-device state was
never created. The file name sorts last so that, in a run stopping at the first failure,
every other test has run before it; it also passes on its own in a fresh process.
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from mordred_b200 import _lib as L
from mordred_b200 import ssb
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

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
    exp, ost = O.q41({k: v.cpu().numpy() for k, v in t.items()}, ssb.DATE_SLOTS)
    assert ost == 0
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
        assert np.array_equal(a, exp), f"call {call} differs from the oracle"
        assert len(ssb.crystal4_groups(a)) > 0


def test_noalloc_rejects_supplier_table_beyond_scratch():
    lib = L.lib()
    big = 262_144 + 1
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = ssb._p(dummy)
    rc = lib.mb_q41_probe_noalloc(p, p, p, p, p, p, 4, p, 4, p, big, p, 4, p, 4, p, None, ssb._stream())
    assert rc == 6  # MB_ERR_SIZE
    assert "size" in lib.mb_error_string(rc).decode()


_FRESH = r"""
import json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
from mordred_b200 import _lib as L, ssb
from oracle import oracle as O
torch.cuda.set_device(0)
s = ssb.Sizes(lo_len=1_000_003, s_len=40_000, c_len=600_000, p_len=1_000_000)
h = ssb.gen_host(s, 77, ssb.QB_FACT, ssb.QB_DIMS)          # host generator: no device state
ht = {"s": np.zeros(s.s_len, np.int32), "c": np.zeros(2 * s.c_len, np.int32),
      "p": np.zeros(s.p_len, np.int32), "d": np.zeros(2 * ssb.DATE_SLOTS, np.int32)}
O.build_ht(h["s_region"], 0, 1, 0, h["s_suppkey"], None, ht["s"], s.s_len, 0, 0)
O.build_ht(h["c_region"], 0, 1, 0, h["c_custkey"], h["c_nation"], ht["c"], s.c_len, 0, 1)
O.build_ht(h["p_mfgr"], 2, 0, 1, h["p_partkey"], None, ht["p"], s.p_len, 0, 0)
O.build_ht(None, 0, 0, 0, h["d_datekey"], h["d_year"], ht["d"], ssb.DATE_SLOTS, ssb.DATE_MIN, 1)
d = {k: torch.from_numpy(v).cuda() for k, v in list(h.items()) + [("ht_" + k, v) for k, v in ht.items()]}
res = torch.zeros(4 * ssb.QB_GROUPS, dtype=torch.int32, device="cuda")
status = torch.zeros(1, dtype=torch.int32, device="cuda")
lib = L.lib()
before = lib.mb_device_state_ready(0)
rcs = []
for _ in range(2):
    res.zero_()
    rcs.append(lib.mb_q41_probe_noalloc(d["lo_orderdate"].data_ptr(), d["lo_partkey"].data_ptr(),
                                        d["lo_custkey"].data_ptr(), d["lo_suppkey"].data_ptr(),
                                        d["lo_revenue"].data_ptr(), d["lo_supplycost"].data_ptr(), s.lo_len,
                                        d["ht_p"].data_ptr(), s.p_len, d["ht_s"].data_ptr(), s.s_len,
                                        d["ht_c"].data_ptr(), s.c_len, d["ht_d"].data_ptr(), ssb.DATE_SLOTS,
                                        res.data_ptr(), status.data_ptr(), ssb._stream()))
torch.cuda.synchronize()
exp, ost = O.q41(h, ssb.DATE_SLOTS)
print(json.dumps({"before": before, "after": lib.mb_device_state_ready(0), "rcs": rcs, "status": int(status.item()),
                  "equal": bool(np.array_equal(res.cpu().numpy(), exp)), "oracle_status": ost,
                  "groups": len(ssb.crystal4_groups(exp))}))
"""


def test_noalloc_in_fresh_process_creates_no_allocating_state():
    """Only the allocation-free entry point runs in this process: the library's per-device
    state (whose set-up cudaMalloc's the status word) must not exist afterwards, and both
    calls must equal the oracle."""
    out = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert r["rcs"] == [0, 0] and r["status"] == 0 and r["oracle_status"] == 0
    assert r["before"] == 0 and r["after"] == 0, r
    assert r["equal"] and r["groups"] > 0
