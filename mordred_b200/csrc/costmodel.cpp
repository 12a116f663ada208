// costmodel.cpp — the analytic cost model of the reference's optimizer and the segment
// placement both planners share.
//
// Analytic model (src/gpudb/CostModel.h:4-6, CostModel.cu:283-440): an operator
// pipeline over L rows costs bytes / bandwidth, with BW_CPU = 42e6 and BW_PCI = 12e6
// bytes per ms and 64-byte cache lines for random accesses. A filter scans 4 B/row; a
// probe scans 4 B/row and touches one cache line per row; a group-by touches one line
// per aggregate column and one for the group; an operator that starts from rows
// materialised on the other device first reads their offsets (one more line per row);
// each operator leaves L * selectivity rows. GPU operators cost nothing when the whole
// pipeline runs on the GPU (CostModel.cu:341-343); moving rows between devices costs
// L * 4 * M / BW_PCI for M columns (transfer_cost, :386-390). mb_cost_calculate restates
// calculate_cost (:283-363) for one placement of a filter/probe/group pipeline; the
// per-segment estimates the planner uses are its all-CPU form and, for the GPU, the
// transfer of the segment's columns that are not resident in the segment cache.
//
// Placement: given per-segment CPU and GPU time estimates (from this model or from the
// learned one), segments go to the device where they finish the query soonest. CPU and
// GPU work on their shares concurrently, so the query takes about max(fixed CPU ms +
// sum of CPU ms, fixed GPU ms + sum of GPU ms), a device's fixed cost (its hash-table
// builds, its launches) paid only when it takes a segment; mb_place_segments orders
// segments by their GPU/CPU time ratio and picks the split point of that order that
// minimises this makespan (the optimum for two machines when each segment's times are
// proportional along the order, and a good heuristic otherwise).
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "mordred_b200.h"

namespace {

constexpr double kBwCpu = 42000000.0;  // bytes per ms (CostModel.h:5)
constexpr double kBwPci = 12000000.0;  // bytes per ms (CostModel.h:6)
constexpr double kLine = 64.0;         // CostModel.h:4

struct Model {
  double L;
  int n_aggr;
  double filter(double sel, bool mat_start) {
    const double scan = mat_start ? L * 4 / kBwCpu + L * kLine / kBwCpu : L * 4 / kBwCpu;
    L *= sel;
    return scan;
  }
  double probe(double sel, bool mat_start) {
    const double scan = mat_start ? L * 4 / kBwCpu + L * kLine / kBwCpu : L * 4 / kBwCpu;
    const double probe_time = L * kLine / kBwCpu;
    L *= sel;
    return scan + probe_time;
  }
  double group(bool mat_start) {
    const double scan = mat_start ? L * 4 / kBwCpu + L * kLine * n_aggr / kBwCpu : L * kLine * n_aggr / kBwCpu;
    return scan + L * kLine / kBwCpu;
  }
  double transfer(int m) const { return L * 4 * m / kBwPci; }
};

bool valid(const mb_cost_pipeline* p) {
  return p && p->num_filters >= 0 && p->num_filters <= MB_MAX_FILTERS && p->num_probes >= 0 &&
         p->num_probes <= MB_MAX_PROBES && p->num_aggr >= 0;
}

}  // namespace

extern "C" double mb_cost_calculate(const mb_cost_pipeline* p, const int* on_gpu, double rows) {
  if (!valid(p) || on_gpu == nullptr || rows < 0) return -1.0;
  const int nf = p->num_filters, np = p->num_probes;
  const bool group_gpu = p->group_by && on_gpu[nf + np];
  const bool group_cpu = p->group_by && !on_gpu[nf + np];
  bool sel_gpu = false, join_gpu = false, sel_cpu = false, join_cpu = false;
  int n_join_gpu = 0;
  for (int f = 0; f < nf; ++f) (on_gpu[f] ? sel_gpu : sel_cpu) = true;
  for (int q = 0; q < np; ++q) {
    if (on_gpu[nf + q]) {
      join_gpu = true;
      ++n_join_gpu;
    } else {
      join_cpu = true;
    }
  }
  Model m{rows, p->num_aggr};
  double cost = 0;
  bool from_gpu = false;
  if (sel_gpu || join_gpu) {
    for (int f = 0; f < nf; ++f)
      if (on_gpu[f]) m.L *= p->filter_sel[f];
    for (int q = 0; q < np; ++q)
      if (on_gpu[nf + q]) m.L *= p->probe_sel[q];
    if (sel_cpu || join_cpu || group_cpu) {
      cost += m.transfer(n_join_gpu + 1);
      from_gpu = true;
    }
  }
  for (int f = 0; f < nf; ++f) {
    if (on_gpu[f]) continue;
    cost += m.filter(p->filter_sel[f], from_gpu);
    from_gpu = false;
  }
  for (int q = 0; q < np; ++q) {
    if (on_gpu[nf + q]) continue;
    cost += m.probe(p->probe_sel[q], from_gpu);
    from_gpu = false;
  }
  if (group_cpu) {
    cost += m.group(from_gpu);
    from_gpu = false;
  }
  if (group_gpu && (sel_cpu || join_cpu))
    cost += m.group(false);
  else if (group_gpu && (sel_gpu || join_gpu))
    cost = 0;
  return cost;
}

extern "C" double mb_cost_cpu_ms(const mb_cost_pipeline* p, double rows) {
  int dev[MB_MAX_FILTERS + MB_MAX_PROBES + 1] = {0};
  return mb_cost_calculate(p, dev, rows);
}

extern "C" double mb_cost_transfer_ms(double rows, int columns) {
  if (rows < 0 || columns < 0) return -1.0;
  return rows * 4.0 * columns / kBwPci;
}

extern "C" double mb_cost_build_ms(double dim_rows) {
  // CostModel.cu:427-440 build_cost without a materialised start: scan + one line per row
  if (dim_rows < 0) return -1.0;
  return dim_rows * 4 / kBwCpu + dim_rows * kLine / kBwCpu;
}

extern "C" int mb_cost_segments(const mb_cost_pipeline* p, int n, const double* rows, const double* first_filter_sel,
                                const int* missing_cols, double* cpu_ms, double* gpu_ms) {
  if (!valid(p) || n < 0 || (n > 0 && (rows == nullptr || cpu_ms == nullptr || gpu_ms == nullptr)))
    return MB_ERR_ARG;
  mb_cost_pipeline q = *p;
  for (int i = 0; i < n; ++i) {
    if (first_filter_sel && q.num_filters > 0) q.filter_sel[0] = first_filter_sel[i];
    cpu_ms[i] = mb_cost_cpu_ms(&q, rows[i]);
    gpu_ms[i] = mb_cost_transfer_ms(rows[i], missing_cols ? missing_cols[i] : 0);
  }
  return MB_OK;
}

extern "C" int mb_place_segments(int n, const double* cpu_ms, const double* gpu_ms, double cpu_fixed_ms,
                                 double gpu_fixed_ms, unsigned char* on_gpu, double* makespan_ms) {
  if (n < 0 || (n > 0 && (cpu_ms == nullptr || gpu_ms == nullptr || on_gpu == nullptr))) return MB_ERR_ARG;
  if (n == 0) {
    if (makespan_ms) *makespan_ms = 0;
    return MB_OK;
  }
  cpu_fixed_ms = std::max(cpu_fixed_ms, 0.0);
  gpu_fixed_ms = std::max(gpu_fixed_ms, 0.0);
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  auto ratio = [&](int i) {
    const double c = std::max(cpu_ms[i], 1e-9), g = std::max(gpu_ms[i], 0.0);
    return g / c;
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ratio(a) < ratio(b); });
  // GPU takes order[0..k), CPU the rest; k = n .. 0
  // a device that takes any segment pays its fixed cost (builds, launches) once
  std::vector<double> suffix_cpu(n + 1, 0.0);
  for (int i = n - 1; i >= 0; --i) suffix_cpu[i] = suffix_cpu[i + 1] + std::max(cpu_ms[order[i]], 0.0);
  double gpu = 0, best = suffix_cpu[0] + cpu_fixed_ms;
  int best_k = 0;
  for (int k = 1; k <= n; ++k) {
    gpu += std::max(gpu_ms[order[k - 1]], 0.0);
    const double span = std::max(gpu + gpu_fixed_ms, k < n ? suffix_cpu[k] + cpu_fixed_ms : 0.0);
    if (span < best) {
      best = span;
      best_k = k;
    }
  }
  for (int i = 0; i < n; ++i) on_gpu[order[i]] = i < best_k ? 1 : 0;
  if (makespan_ms) *makespan_ms = best;
  return MB_OK;
}
