"""Batched execution over the host-resident segmented table (mordred_b200.batch_engine):
every query of a window, under every placement (all GPU with resident and staged
segments, all CPU, the planners' own splits), equals the oracle running it alone over the
whole table, and the one-query-at-a-time executor's result. CPU part: the window planning
helpers."""
import numpy as np
import pytest

from mordred_b200 import batch as B
from mordred_b200 import ssb

pytestmark = pytest.mark.gpu


class _Fixed:
    """A planner that prices every segment so that all go to one device."""

    def __init__(self, name, gpu):
        self.name, self.gpu = name, gpu

    def predict_many(self, ctxs):
        out = []
        for c in ctxs:
            n = len(c)
            cpu_ms = np.full(n, 1e6 if self.gpu else 1.0)
            gpu_ms = np.full(n, 1.0 if self.gpu else 1e6)
            out.append((cpu_ms, gpu_ms, 0.0, 0.0))
        return out

    def predict(self, ctx):
        return self.predict_many([ctx])[0]


@pytest.fixture(scope="module")
def table():
    import torch
    from mordred_b200 import _lib as L
    from mordred_b200.engine import SegmentedTable
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    # 14 segments of 2**20 rows and a partial one; dimension sizes below the workload's
    return SegmentedTable(14 * (1 << 20) + 123_457, 2718, ssb.Sizes(lo_len=14 * (1 << 20) + 123_457, s_len=4_000,
                                                                     c_len=60_000, p_len=100_000))


def _host(t):
    h = dict(t.host)
    h.update(t.hdims)
    return h


def test_windows_equal_oracle_and_one_at_a_time(table):
    from mordred_b200 import _lib as L
    from mordred_b200.batch_engine import BatchExecutor
    from mordred_b200.engine import Executor
    from mordred_b200.planner import AnalyticPlanner
    from query_oracle import expected
    qs = B.generate_queries(60, seed=404, sel_lo=1e-4, sel_hi=0.3)
    h = _host(table)
    exp = [expected(h, table.sizes, q).view(np.int32) for q in qs]
    # small cache: 20 managed slots + 2 x 2 staged segments of 9 columns
    ex = BatchExecutor(table, cache_slots=20 + 2 * 2 * 9, stage_segments=2)
    for planner in (_Fixed("gpu", True), _Fixed("cpu", False), AnalyticPlanner()):
        runs = ex.run(qs, planner, window=25)
        got = [r for w in runs for r in w.results]
        for i, (g, e) in enumerate(zip(got, exp)):
            assert np.array_equal(g, e), (planner.name, i, qs[i].template)
        if planner.name == "gpu":
            assert sum(w.staged_segments for w in runs) > 0 and sum(w.cpu_segments for w in runs) == 0
        if planner.name == "cpu":
            assert sum(w.gpu_segments for w in runs) == 0
    # the one-query-at-a-time executor agrees
    ex.close()
    one = Executor(table, cache_slots=40)
    for i, q in enumerate(qs[:20]):
        assert np.array_equal(one.run(q, AnalyticPlanner()).result, exp[i])
    assert L.device_status(0) == 0


def test_admission_keeps_demanded_segments_resident(table):
    from mordred_b200.batch_engine import BatchExecutor
    from mordred_b200.planner import AnalyticPlanner
    import dataclasses
    ex = BatchExecutor(table, cache_slots=60 + 2 * 2 * 9, stage_segments=2)
    # every window reads the first two months only: those segments become resident
    qs = [dataclasses.replace(q, date=(19920105, 19920225)) for q in B.generate_queries(30, seed=9)]
    runs = ex.run(qs, AnalyticPlanner(), window=10)
    ex.close()
    assert runs[0].copied_column_segments > 0
    assert all(w.staged_segments == 0 for w in runs[1:])


def test_one_window_of_several_launch_chunks(table):
    """A window of 300 queries (two 256-query launch chunks, each scanning only the
    segments its queries can match) equals the oracle query by query, all on the GPU and
    under the analytic planner's split."""
    from mordred_b200 import _lib as L
    from mordred_b200.batch_engine import BatchExecutor
    from mordred_b200.planner import AnalyticPlanner
    from query_oracle import expected
    qs = B.generate_queries(300, seed=707, sel_lo=1e-4, sel_hi=0.3)
    h = _host(table)
    exp = [expected(h, table.sizes, q).view(np.int32) for q in qs]
    ex = BatchExecutor(table, cache_slots=40 + 2 * 2 * 9, stage_segments=2)
    for planner in (_Fixed("gpu", True), AnalyticPlanner()):
        runs = ex.run(qs, planner, window=len(qs))
        assert len(runs) == 1 and runs[0].launches >= 2
        for i, (g, e) in enumerate(zip(runs[0].results, exp)):
            assert np.array_equal(g, e), (planner.name, i, qs[i].template)
    ex.close()
    assert L.device_status(0) == 0
