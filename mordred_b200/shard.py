"""Row-sharded execution over several GPUs: rank r of N holds fact rows [r*n, (r+1)*n)
of one table (the seeded generator takes a row offset, so every shard is a slice of the
same table) and replicated dimension tables; the only exchange is one all-reduce of the
queries' dense group sums (64-bit integer sums are exact in any order). The reference
has no multi-GPU path; star queries over independent fact rows partition this way.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from . import _lib as L
from . import ssb


def gen_shard(sizes: ssb.Sizes, seed: int, names: list[str], rank: int, n: int, device="cuda") -> dict:
    """This rank's rows [rank*n, (rank+1)*n) of the named fact columns (device or "cpu")."""
    out = {}
    if str(device) == "cpu":
        for name in names:
            t = torch.empty(n, dtype=torch.int32)
            L.call("mb_gen_fact_column_host", ssb.FACT_COLUMNS[name], seed, rank * n, n, sizes.s_len, sizes.c_len,
                   sizes.p_len, t.data_ptr(), 0)
            out[name] = t
        return out
    st = ssb._stream()
    for name in names:
        t = torch.empty(n, dtype=torch.int32, device=device)
        L.call("mb_gen_fact_column", ssb.FACT_COLUMNS[name], seed, rank * n, n, sizes.s_len, sizes.c_len, sizes.p_len,
               t.data_ptr(), st)
        out[name] = t
    return out


def crystal4_sums(res: torch.Tensor) -> torch.Tensor:
    """The 64-bit group sums of an int[4*G] result (words 2-3 of each group), as int64[G]."""
    return res.view(-1, 4)[:, 2:4].contiguous().view(torch.int64).view(-1)


def allreduce_sums(parts: list[torch.Tensor], out: torch.Tensor) -> torch.Tensor:
    """Concatenate the ranks' dense sums into `out` and sum them over all ranks in place."""
    off = 0
    for p in parts:
        out[off: off + p.numel()].copy_(p)
        off += p.numel()
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(out)
    return out
