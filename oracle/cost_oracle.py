"""Python restatement of the reference's analytic cost model, for tests.

TEST INFRASTRUCTURE ONLY: follows src/gpudb/CostModel.cu:283-440 (calculate_cost,
probe_cost, transfer_cost, filter_cost, group_cost) and CostModel.h:4-6 constants, for
a filter -> probe -> group pipeline; the checker of mordred_b200/csrc/costmodel.cpp.
"""
BW_CPU, BW_PCI, CACHE_LINE = 42_000_000.0, 12_000_000.0, 64.0


def calculate_cost(filter_sel, probe_sel, group_by, n_aggr, on_gpu, rows):
    nf, np_ = len(filter_sel), len(probe_sel)
    sel_gpu = [s for s, g in zip(filter_sel, on_gpu[:nf]) if g]
    sel_cpu = [s for s, g in zip(filter_sel, on_gpu[:nf]) if not g]
    join_gpu = [s for s, g in zip(probe_sel, on_gpu[nf:nf + np_]) if g]
    join_cpu = [s for s, g in zip(probe_sel, on_gpu[nf:nf + np_]) if not g]
    group_gpu = group_by and on_gpu[nf + np_]
    group_cpu = group_by and not on_gpu[nf + np_]
    L = float(rows)
    cost, from_gpu = 0.0, False
    if sel_gpu or join_gpu:
        for s in sel_gpu + join_gpu:
            L *= s
        if sel_cpu or join_cpu or group_cpu:
            cost += L * 4 * (len(join_gpu) + 1) / BW_PCI
            from_gpu = True
    for s in sel_cpu:
        cost += (L * 4 / BW_CPU + L * CACHE_LINE / BW_CPU) if from_gpu else L * 4 / BW_CPU
        from_gpu = False
        L *= s
    for s in join_cpu:
        scan = (L * 4 / BW_CPU + L * CACHE_LINE / BW_CPU) if from_gpu else L * 4 / BW_CPU
        cost += scan + L * CACHE_LINE / BW_CPU
        from_gpu = False
        L *= s
    if group_cpu:
        scan = (L * 4 / BW_CPU + L * CACHE_LINE * n_aggr / BW_CPU) if from_gpu else L * CACHE_LINE * n_aggr / BW_CPU
        cost += scan + L * CACHE_LINE / BW_CPU
    if group_gpu and (sel_cpu or join_cpu):
        cost += L * CACHE_LINE * n_aggr / BW_CPU + L * CACHE_LINE / BW_CPU
    elif group_gpu and (sel_gpu or join_gpu):
        cost = 0.0
    return cost
