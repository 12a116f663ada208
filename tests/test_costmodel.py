"""The analytic cost model against its restatement and a hand-computed case, and the
CPU/GPU segment placement against an exhaustive search over its candidate splits."""
import ctypes as C
import itertools

import numpy as np
import pytest

from mordred_b200 import _lib as L
from oracle import cost_oracle as CO


def _pipe(fs, ps, group_by=1, n_aggr=2):
    p = L.MbCostPipeline()
    p.num_filters, p.num_probes, p.group_by, p.num_aggr = len(fs), len(ps), group_by, n_aggr
    for i, s in enumerate(fs):
        p.filter_sel[i] = s
    for i, s in enumerate(ps):
        p.probe_sel[i] = s
    return p


def test_segment_batch_and_build_cost():
    p = _pipe([0.5, 0.3], [0.2, 1.0], 1, 2)
    rows = np.array([1e6, 5e5, 1048576.0])
    sel = np.array([0.1, 1.0, 0.0])
    miss = np.array([0, 3, 6], np.int32)
    cpu_ms, gpu_ms = np.zeros(3), np.zeros(3)
    L.call("mb_cost_segments", C.byref(p), 3, rows.ctypes.data, sel.ctypes.data, miss.ctypes.data, cpu_ms.ctypes.data,
           gpu_ms.ctypes.data)
    for i in range(3):
        assert abs(cpu_ms[i] - CO.calculate_cost([sel[i], 0.3], [0.2, 1.0], 1, 2, [0] * 5, rows[i])) < 1e-12
        assert abs(gpu_ms[i] - rows[i] * 4 * miss[i] / 12e6) < 1e-12
    assert abs(L.lib().mb_cost_build_ms(1e6) - (1e6 * 4 + 1e6 * 64) / 42e6) < 1e-12


def test_hand_computed_all_cpu():
    # 1e6 rows: filter 0.3 keeps 3e5; probe 0.2 keeps 6e4; group over 2 aggregate columns
    p = _pipe([0.3], [0.2])
    exp = 1e6 * 4 / 42e6 + (3e5 * 4 / 42e6 + 3e5 * 64 / 42e6) + (6e4 * 64 * 2 / 42e6 + 6e4 * 64 / 42e6)
    assert abs(L.lib().mb_cost_cpu_ms(C.byref(p), 1e6) - exp) < 1e-12
    assert abs(L.lib().mb_cost_transfer_ms(1e6, 3) - 1e6 * 12 / 12e6) < 1e-12


def test_every_placement_matches_restatement():
    rng = np.random.default_rng(0)
    for _ in range(40):
        fs = list(rng.uniform(0.01, 1, rng.integers(0, 4)))
        ps = list(rng.uniform(0.01, 1, rng.integers(0, 5)))
        g = int(rng.integers(0, 2))
        p = _pipe(fs, ps, g, int(rng.integers(1, 3)))
        nops = len(fs) + len(ps) + 1
        for dev in itertools.product([0, 1], repeat=nops):
            arr = (C.c_int * nops)(*dev)
            got = L.lib().mb_cost_calculate(C.byref(p), arr, 2.5e6)
            exp = CO.calculate_cost(fs, ps, g, p.num_aggr, list(dev), 2.5e6)
            assert abs(got - exp) <= 1e-9 * max(1.0, abs(exp)), (fs, ps, g, dev)


def _span(cpu, gpu, on, cf, gf):
    g = gpu[on].sum() + (gf if on.any() else 0.0)
    c = cpu[~on].sum() + (cf if (~on).any() else 0.0)
    return max(g, c)


@pytest.mark.parametrize("n", [0, 1, 2, 7, 40])
@pytest.mark.parametrize("fixed", [(0.0, 0.0), (2.0, 0.3)])
def test_placement_is_best_split_of_ratio_order(n, fixed):
    cf, gf = fixed
    rng = np.random.default_rng(n)
    cpu = rng.uniform(0.1, 5, n)
    gpu = rng.uniform(0.0, 3, n)
    on = np.zeros(n, np.uint8)
    span = C.c_double(0)
    L.call("mb_place_segments", n, cpu.ctypes.data, gpu.ctypes.data, cf, gf, on.ctypes.data, C.byref(span))
    on = on.astype(bool)
    got = _span(cpu, gpu, on, cf, gf) if n else 0.0
    assert abs(got - span.value) < 1e-9
    order = np.argsort(gpu / cpu, kind="stable")
    best = 0.0
    if n:
        best = min(_span(cpu, gpu, np.isin(np.arange(n), order[:k]), cf, gf) for k in range(n + 1))
    assert abs(span.value - best) < 1e-9
    if n <= 10 and n > 0:  # and near the true optimum over all 2^n assignments
        opt = min(_span(cpu, gpu, np.array(m, bool), cf, gf) for m in itertools.product([0, 1], repeat=n))
        assert span.value <= opt + max(gpu.max(), cpu.max())


def test_features_many_equals_per_query_features():
    """The planner's stacked feature builder equals features() query by query."""
    import numpy as np
    from mordred_b200.planner import QueryContext, features, features_many
    rng = np.random.default_rng(4)
    ctxs = []
    for k in range(40):
        n = int(rng.integers(0, 30))
        tpl = ("agg", "qa", "qb")[k % 3]
        ctxs.append(QueryContext(tpl, rng.integers(1, 1 << 20, n).astype(np.float64), rng.random(n),
                                 {x: float(rng.random()) for x in ("discount", "quantity", "s", "c", "p")},
                                 {"agg": 4, "qa": 4, "qb": 6}[tpl], rng.integers(0, 5, n).astype(np.int32),
                                 int(rng.integers(0, 1 << 24)), 1000, {"agg": 1, "qa": 7000, "qb": 175}[tpl],
                                 16, float(rng.random())))
    want = np.concatenate([features(c) for c in ctxs if len(c)])
    got = features_many(ctxs)
    assert got.shape == want.shape
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6)
