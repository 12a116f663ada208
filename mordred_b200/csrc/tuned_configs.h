// tuned_configs.h — launch configuration defaults of the fused star kernel per query
// shape, written by mordred_b200/autotune.py from sweeps on a B200 (threads x rows per
// thread x stages x group mode, 120,000,000-row fact table). A shape is keyed by its
// filter count, probe count, first probe's table layout, whether it groups, and whether
// its group array is large (> 2,048 groups); an entry with max_rows > 0 applies only to
// calls of at most that many rows and is looked up first (small tables: 6,000,000 rows
// swept over 20 separate tables replayed back to back from a CUDA graph). Unknown shapes
// take kDefaultConfig.
#pragma once

namespace mb {

struct TunedConfig {
  int threads, items, stages, group_mode;
  int mirrors = 0;  // 1: large calls of this shape use cluster-resident mirrors by default
  int pack = 0;     // 1: the variant that packs the first sparse probe's survivors across the warp;
                    // 2: packed, returning each stage before its last batch's probes; 3: unpacked,
                    // with that early return
};

struct TunedEntry {
  int nf, np, p0_layout, grouped, big_groups;
  TunedConfig cfg;
  long long max_rows = 0;  // > 0: only for calls of at most this many rows
};

static const TunedConfig kDefaultConfig = {256, 8, 2, 0};

static const TunedEntry kTuned[] = {
    {3, 0, -1, 0, 0, {128, 16, 2, 0}, 16ll << 20},  // filter-aggregate, 6 M rows: 0.0189 ms, 5.08 TB/s
    {3, 0, -1, 0, 0, {256, 16, 4, 0}},  // filter-aggregate (q11 form): 0.2684 ms, 7.15 TB/s
    {0, 3, 0, 1, 1, {768, 8, 3, 2, 0, 3}},  // Query A form: 0.4558 ms, 4.21 TB/s (24 warps, early stage return)
    {0, 4, 0, 1, 0, {768, 8, 2, 1, 0, 2}},  // Query B form: 0.5942 ms, 4.85 TB/s (24 warps, packed, early stage return)
    {0, 4, 2, 1, 0, {768, 8, 2, 1, 0, 2}},  // engine four-table group-by: 0.6432 ms, 4.48 TB/s (24 warps, packed, early return)
};

inline TunedConfig tuned_config(int nf, int np, int p0_layout, int res_layout, int total_val, long long rows) {
  const int grouped = res_layout != 0 ? 1 : 0;
  const int big = grouped && total_val > 2048 ? 1 : 0;
  const int l0 = np > 0 ? p0_layout : -1;
  for (const TunedEntry& e : kTuned)
    if (e.nf == nf && e.np == np && e.p0_layout == l0 && e.grouped == grouped && e.big_groups == big &&
        (e.max_rows == 0 || rows <= e.max_rows))
      return e.cfg;
  TunedConfig c = kDefaultConfig;
  if (big) c.group_mode = 2;  // large group arrays: L2 atomics keep shared memory for stages
  return c;
}

}  // namespace mb
