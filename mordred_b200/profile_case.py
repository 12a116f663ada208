"""Run the workload's queries a few times on a chosen table size, for profilers.

    python -m mordred_b200.profile_case [--rows N] [--reps K]

Runs the filter-aggregate (mb_q11_query), Query A (builds + mb_q21_probe) and Query B
(builds + mb_q41_probe) through the C ABI with the tuned launch defaults, K times each,
then checks the device status word. Small sizes (for example 24,000,000 rows: 576 MB
of fact columns, above the 126 MB L2) keep an ncu capture short.
"""
from __future__ import annotations

import argparse

import torch

from . import _lib as L
from . import ssb


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=24_000_000)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--batch", type=int, default=0, help="run a batch of this many generated queries instead")
    args = ap.parse_args()
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    s = ssb.Sizes(lo_len=args.rows)
    if args.batch:
        from . import batch as B
        t = ssb.gen_device(s, args.seed, B.BATCH_FACT, B.BATCH_DIMS)
        pats = B.build_pats(t, s)
        qs = B.generate_queries(args.batch, seed=args.seed)
        res = [q.result_buffer() for q in qs]
        for _ in range(args.reps):
            B.run_batch(t, pats, qs, res, args.rows)
        torch.cuda.synchronize()
        st = L.device_status(0)
        if st:
            raise SystemExit(f"device status {st:#x}")
        print(f"ok: {args.reps} x batch of {args.batch} queries over {args.rows:,} rows")
        return
    t = ssb.gen_device(s, args.seed, ssb.QB_FACT + ["lo_discount", "lo_quantity", "lo_extendedprice"],
                       sorted(set(ssb.QA_DIMS + ssb.QB_DIMS)))
    ws = ssb.StarWorkspace(s)
    for _ in range(args.reps):
        ssb.q11(t, args.rows, ws)
        ssb.query_a(t, ws)
        ssb.query_b(t, ws)
    torch.cuda.synchronize()
    st = L.device_status(0)
    if st:
        raise SystemExit(f"device status {st:#x}")
    print(f"ok: {args.reps} x (q11, Query A, Query B) over {args.rows:,} rows; "
          f"{L.launch_count()} library launches")


if __name__ == "__main__":
    main()
