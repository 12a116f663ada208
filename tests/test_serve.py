"""Serving loop: the admission controller (CPU) and the real-time server (GPU)."""
import numpy as np
import pytest

from mordred_b200 import batch as B
from mordred_b200 import serve as S


def test_admission_fifo_under_budget():
    ac = S.AdmissionController(budget_bytes=10_000, max_queue=5)
    assert ac.arrive(0, 4096) and ac.arrive(1, 4096)
    assert ac.arrive(2, 4096)            # does not fit yet: waits
    assert [q for q, _ in ac.admitted] == [0, 1] and [q for q, _ in ac.waiting] == [2]
    assert not ac.arrive(3, 20_000)      # larger than the whole budget: rejected
    assert ac.arrive(4, 1000)            # fits, but waits behind 2: arrival order is kept
    assert [q for q, _ in ac.waiting] == [2, 4]
    got = ac.take(8)
    assert [q for q, _ in got] == [0, 1] and ac.held == 8192
    ac.release(4096)
    assert [q for q, _ in ac.admitted] == [2, 4] and ac.held == 4096 + 4096 + 1000
    assert ac.arrive(5, 10) and ac.arrive(6, 10) and ac.arrive(7, 10)
    assert not ac.arrive(8, 10)          # queue limit (five queued)
    assert ac.rejected == 2 and ac.deferred > 0


def test_poisson_arrivals_rate():
    a = S.poisson_arrivals(2000.0, 20_000, 1)
    assert np.all(np.diff(a) > 0)
    assert abs(20_000 / a[-1] - 2000.0) < 60


def test_query_bytes_fit_in_budget():
    qs = B.generate_queries(300, seed=2)
    total = sum(S.query_bytes(q) for q in qs)
    assert 0 < total < (16 << 30)
    assert all(S.query_bytes(q) % 4096 == 0 for q in qs)


@pytest.mark.gpu
def test_server_answers_every_query_exactly():
    import torch
    from mordred_b200 import _lib as L
    from mordred_b200 import ssb
    torch.cuda.set_device(0)
    n = 3_000_001
    sizes = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(sizes, 23, B.BATCH_FACT, B.BATCH_DIMS)
    srv = S.Server(t, sizes, n, budget_bytes=4 << 20, max_batch=64)
    qs = B.generate_queries(300, seed=4, sel_lo=1e-4, sel_hi=0.3)
    arr = S.poisson_arrivals(3000.0, len(qs), 6)
    rep, res = srv.serve(qs, arr, keep_results=True)
    s = rep.summary(n)
    assert s["completed"] == 300 and s["rejected"] == 0 and rep.batches >= 5
    assert max(rep.batch_sizes) <= 64 and rep.peak_held_bytes <= 4 << 20
    assert all(x > 0 for x in rep.latencies_ms)
    ws = B.AloneWorkspace(sizes)
    for qid in range(0, 300, 23):
        r = qs[qid].result_buffer()
        B.run_alone(t, ws, qs[qid], r, n)
        exp = r.cpu().numpy()
        assert np.array_equal(res[qid].reshape(-1), exp.reshape(-1)), qid
    assert L.device_status(0) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("chunks", [1, 5])
def test_circular_server_answers_every_query_exactly(chunks):
    """Queries that join a circular scan between chunks get exactly the results of
    running alone, whatever chunk they joined at."""
    import torch
    from mordred_b200 import _lib as L
    from mordred_b200 import ssb
    torch.cuda.set_device(0)
    n = 3_000_001
    sizes = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(sizes, 29, B.BATCH_FACT, B.BATCH_DIMS)
    srv = S.CircularServer(t, sizes, n, budget_bytes=4 << 20, max_active=64, chunks=chunks, burst_active=64)
    assert len(srv.bounds) == chunks and srv.bounds[-1][1] == n
    qs = B.generate_queries(300, seed=5, sel_lo=1e-4, sel_hi=0.3)
    arr = S.poisson_arrivals(3000.0, len(qs), 7)
    rep, res = srv.serve(qs, arr, keep_results=True)
    s = rep.summary(n)
    assert s["completed"] == 300 and s["rejected"] == 0
    assert max(rep.batch_sizes) <= 64 and rep.peak_held_bytes <= 4 << 20
    assert all(x > 0 for x in rep.latencies_ms)
    ws = B.AloneWorkspace(sizes)
    for qid in range(0, 300, 7):
        r = qs[qid].result_buffer()
        B.run_alone(t, ws, qs[qid], r, n)
        assert np.array_equal(res[qid].reshape(-1), r.cpu().numpy().reshape(-1)), qid
    assert L.device_status(0) == 0


@pytest.mark.gpu
def test_circular_server_skips_chunks_outside_a_query_dates():
    """Over a date-sorted table a query joins only the chunks whose orderdate range meets
    its own; queries needing one chunk, several, or none all get their results alone."""
    import dataclasses

    import torch
    from mordred_b200 import _lib as L
    from mordred_b200 import ssb
    from mordred_b200.engine import SegmentedTable
    torch.cuda.set_device(0)
    n = 6 * (1 << 20) + 777
    sizes = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    table = SegmentedTable(n, 37, sizes)
    t = {k: torch.from_numpy(table.host[k]).cuda() for k in B.BATCH_FACT}
    t.update(table.dims)
    t.update(ssb.gen_device(sizes, 37, [], [d for d in B.BATCH_DIMS if d not in t]))
    srv = S.CircularServer(t, sizes, n, budget_bytes=64 << 20, max_active=64, chunks=8)
    qs = B.generate_queries(150, seed=21, sel_lo=1e-4, sel_hi=0.3)
    qs += [dataclasses.replace(q, date=(19990101, 19991231)) for q in qs[:5]]  # no row can match
    need = [int(srv.chunks_needed(q).sum()) for q in qs]
    assert min(need) == 0 and any(k == 1 for k in need) and max(need) > 1
    arr = S.poisson_arrivals(2000.0, len(qs), 23)
    rep, res = srv.serve(qs, arr, keep_results=True)
    assert rep.summary(n)["completed"] == len(qs)
    ws = B.AloneWorkspace(sizes)
    for qid in range(len(qs)):
        r = qs[qid].result_buffer()
        B.run_alone(t, ws, qs[qid], r, n)
        assert np.array_equal(np.asarray(res[qid]).reshape(-1).view(np.int32), r.cpu().numpy().reshape(-1).view(np.int32)), qid
    assert L.device_status(0) == 0


@pytest.mark.gpu
def test_circular_server_raises_its_cap_under_a_backlog():
    """A burst larger than the active-set cap: the cap rises to burst_active while admitted
    queries wait longer than a lap, never beyond it, and every result stays exact."""
    import torch
    from mordred_b200 import _lib as L
    from mordred_b200 import ssb
    torch.cuda.set_device(0)
    n = 2_000_003
    sizes = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    t = ssb.gen_device(sizes, 31, B.BATCH_FACT, B.BATCH_DIMS)
    srv = S.CircularServer(t, sizes, n, budget_bytes=64 << 20, max_active=8, chunks=4, burst_active=40)
    qs = B.generate_queries(240, seed=11, sel_lo=1e-4, sel_hi=0.3)
    # 40 queries at first, then the other 200 all at once after the first laps
    arr = np.concatenate([np.linspace(0.0, 0.002, 40), np.full(200, 0.05)])
    rep, res = srv.serve(qs, arr, keep_results=True)
    assert rep.summary(n)["completed"] == 240
    assert rep.cap_raises >= 1 and max(rep.batch_sizes) <= 40 and max(rep.batch_sizes) > 8
    ws = B.AloneWorkspace(sizes)
    for qid in range(0, 240, 11):
        r = qs[qid].result_buffer()
        B.run_alone(t, ws, qs[qid], r, n)
        assert np.array_equal(res[qid].reshape(-1), r.cpu().numpy().reshape(-1)), qid
    assert L.device_status(0) == 0


class _CheapCpu:
    """A planner stub predicting 0.1 ms of CPU work per segment (routes what it can)."""
    name = "stub"

    def predict(self, ctx):
        n = len(ctx)
        return np.full(n, 0.1), np.full(n, 1.0), 0.2, 0.0


def test_router_prefers_the_gpu_until_it_has_seen_gpu_latencies():
    r = S.PlannerRouter.__new__(S.PlannerRouter)
    r.gpu_lat = __import__("collections").deque(maxlen=64)
    r.considered = 0
    assert not r.route(0, B.generate_queries(1, seed=1)[0])


def test_router_keeps_at_most_max_inflight_queries_on_the_cpu():
    r = S.PlannerRouter.__new__(S.PlannerRouter)
    r.gpu_lat = __import__("collections").deque([300.0] * 16, maxlen=64)
    r.considered = 0
    r.gpu_target_ms = 100.0
    r.max_inflight, r.inflight = 1, 1
    assert not r.route(0, B.generate_queries(1, seed=1)[0])  # busy: never reaches the model


def test_router_keeps_queries_on_the_gpu_while_it_meets_its_latency_target():
    r = S.PlannerRouter.__new__(S.PlannerRouter)
    r.gpu_lat = __import__("collections").deque([30.0] * 16, maxlen=64)
    r.considered = 0
    r.gpu_target_ms = 100.0
    assert not r.route(0, B.generate_queries(1, seed=1)[0])  # never reaches the model


@pytest.mark.gpu
@pytest.mark.parametrize("server", ["whole", "circular"])
def test_router_sends_queries_to_the_cpu_with_exact_results(server):
    """Over a date-sorted resident table, the router answers some queries on the host
    cores (candidate segments only); every query's result equals its run alone."""
    import torch
    from mordred_b200 import _lib as L
    from mordred_b200 import ssb
    from mordred_b200.engine import SegmentedTable
    torch.cuda.set_device(0)
    n = 6 * (1 << 20) + 777
    sizes = ssb.Sizes(lo_len=n, s_len=4_000, c_len=60_000, p_len=100_000)
    table = SegmentedTable(n, 31, sizes)
    t = {k: torch.from_numpy(table.host[k]).cuda() for k in B.BATCH_FACT}
    t.update(table.dims)
    t.update(ssb.gen_device(sizes, 31, [], [d for d in B.BATCH_DIMS if d not in t]))
    srv = S.Server(t, sizes, n, budget_bytes=4 << 20, max_batch=64) if server == "whole" else \
        S.CircularServer(t, sizes, n, budget_bytes=4 << 20, max_active=64, chunks=4)
    qs = B.generate_queries(240, seed=12, sel_lo=1e-4, sel_hi=0.3)
    arr = S.poisson_arrivals(1500.0, len(qs), 13)
    router = S.PlannerRouter(table, _CheapCpu(), margin=1.0, max_backlog_ms=1e9, gpu_target_ms=0.0, max_inflight=8)
    rep, res = srv.serve(qs, arr, keep_results=True, router=router)
    router.close()
    s = rep.summary(n)
    assert s["completed"] == 240 and rep.cpu_answered > 10 and rep.cpu_answered < 240
    ws = B.AloneWorkspace(sizes)
    for qid in range(240):
        r = qs[qid].result_buffer()
        B.run_alone(t, ws, qs[qid], r, n)
        assert np.array_equal(np.asarray(res[qid]).reshape(-1).view(np.int32), r.cpu().numpy().reshape(-1).view(np.int32)), qid
    assert L.device_status(0) == 0
