/*
 * star_oracle.h — CPU oracle for the star-query hot path. TEST INFRASTRUCTURE ONLY:
 * it is the checker the CUDA path is compared against and the CPU baseline that
 * bench.py times; the product never links, imports or calls it.
 *
 * Two families, both plain C with POSIX threads and 64-bit integer sums:
 *  - orc_q11 / orc_q21 / orc_q41 restate the reference's standalone CPU engine
 *    (src/cpu/ssb/q11.cpp:21-70, q21.cpp:32-167, q41.cpp:32-179) with its constants
 *    made parameters;
 *  - orc_build / orc_star restate the engine's CPU operators (build_CPU,
 *    src/gpudb/CPUProcessing.cu:1034-1104, and filter_probe_group_by_CPU,
 *    CPUProcessing.cu:723-866, widened to the Crystal hash layouts and the
 *    result layouts of the GPU kernels) so any fused pipeline the C ABI accepts has a
 *    row-by-row CPU counterpart.
 */
#ifndef MORDRED_STAR_ORACLE_H
#define MORDRED_STAR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_FILTERS 3
#define ORC_MAX_PROBES 4

/* Status bits, numerically equal to the device status bits of the CUDA path. */
#define ORC_PROBE_RANGE 0x1u
#define ORC_GROUP_RANGE 0x2u

typedef struct orc_filter { const int* col; int mode; int c1, c2; } orc_filter;

/* Probe layouts 0 KEY, 1 KEY_VAL, 2 VAL_OFF as in orc_build; 3 = no table, the payload is
 * passed through from an earlier join: payload = ht[fkey[k]] where ht is a dimension column,
 * fkey a dimension-offset list read at list position k, num_slots the dimension's rows
 * (CPUProcessing.cu:905-908, "dim_val1 = gargs.group_col1[offset.h_dim_off1[...]]"). */
#define ORC_LAYOUT_PASS 3

typedef struct orc_probe {
  const int* fkey;
  const int* ht;
  int num_slots, key_min, layout, min_val, unique_val, res_slot;
} orc_probe;

typedef struct orc_star_args {
  int64_t num_rows;
  int num_filters;
  orc_filter filter[ORC_MAX_FILTERS];
  int num_probes;
  orc_probe probe[ORC_MAX_PROBES];
  const int* aggr[2];
  int agg_op, total_val, group_bias, res_layout;
  void* res;                   /* host result in the layout of res_layout, accumulated into */
  unsigned long long* count;   /* optional */
  int count_after;
  /* Segment addressing: when segment_size > 0, row r of the call reads row
   * segment_group[r / segment_size] * segment_size + r % segment_size of each column
   * (CPUProcessing.cu:741,751); without segment_group the segment is
   * (start_offset + r) / segment_size. */
  const short* segment_group;
  int64_t start_offset;
  int segment_size;
  /* Offset-list input (the *_CPU2 forms, CPUProcessing.cu:868-1032): when rows is
   * non-NULL the call visits k in [0, num_rows) and reads every column at the physical
   * row rows[k] (no segment mapping); pass-through probes read their lists at k. */
  const int* rows;
} orc_star_args;

/* Returns ORC_* status bits (0 = clean). nthreads <= 0: all hardware threads. */
unsigned orc_star(const orc_star_args* a, int nthreads);

/* Selection with compaction (filter_probe_CPU / probe_CPU / filter_CPU and their list
 * forms, CPUProcessing.cu:3-437,1158-1333): the rows passing a's filters and probes, in
 * visiting order. lo_off[k] = physical row; dim_off[p] (optional per probe) = the probe's
 * output: VAL_OFF the dimension row ht[2h+1] - 1, KEY_VAL the payload, KEY 0, a
 * pass-through probe its passed offset. Writes at most `capacity` entries, returns the
 * number of passing rows; *status (optional) receives ORC_* bits. Aggregate fields of a
 * are ignored. Sequential. */
int64_t orc_select(const orc_star_args* a, int* lo_off, int* const* dim_off, int64_t capacity,
                   unsigned* status);

/* Filtered PHT build into a zeroed table in `layout` (0 KEY, 1 KEY_VAL, 2 VAL_OFF).
 * filter NULL = no filter; mode 0 EQ, 1 BETWEEN, 2 EQ OR EQ. row ids for VAL_OFF are
 * row_base + i. presence (optional) receives the slot bitmap. Sequential, row order. */
unsigned orc_build(const int* filter, int mode, int c1, int c2, const int* key, const int* val,
                   int64_t n, int* ht, int num_slots, int key_min, int layout, int64_t row_base,
                   uint32_t* presence);

/* Engine builds over a dimension-offset list or with the key range (build_CPU2,
 * build_CPU_minmax, build_CPU_minmax2: CPUProcessing.cu:1106-1156,1821-1994): rows
 * (optional) lists the dimension rows to build from (row id = rows[k]); otherwise rows
 * row_base + i. Layout VAL_OFF. minmax (optional, int[2]) folds in the min and max key of
 * the rows that pass the filter, starting from {val_max, val_min} as the reference's
 * per-task accumulators do. */
unsigned orc_build_rows(const int* filter, int mode, int c1, int c2, const int* key, const int* val,
                        const int* rows, int64_t n, int* ht, int num_slots, int key_min, int64_t row_base,
                        int* minmax, int val_min, int val_max);

/* src/cpu/ssb/q11.cpp:21-70 with the predicate constants as parameters. */
unsigned long long orc_q11(const int* lo_orderdate, const int* lo_discount, const int* lo_quantity,
                           const int* lo_extendedprice, int64_t n, int date_lo_excl, int date_hi_excl,
                           int disc_lo, int disc_hi, int qty_lt, int nthreads);

/* src/cpu/ssb/q21.cpp:32-167. res: int[6 * 7000], {year, brand, u64 revenue at +2}.
 * d_val_len = number of date slots (the reference uses 61130; 61131 covers 19981231). */
unsigned orc_q21(const int* lo_orderdate, const int* lo_partkey, const int* lo_suppkey,
                 const int* lo_revenue, int64_t lo_len, const int* p_partkey, const int* p_brand1,
                 const int* p_category, int p_len, const int* d_datekey, const int* d_year, int d_len,
                 const int* s_suppkey, const int* s_region, int s_len, int d_val_len, int category,
                 int region, int* res, int nthreads);

/* src/cpu/ssb/q41.cpp:32-179. res: int[4 * 175], {year, c_nation, u64 profit at +2}. */
unsigned orc_q41(const int* lo_orderdate, const int* lo_custkey, const int* lo_partkey,
                 const int* lo_suppkey, const int* lo_revenue, const int* lo_supplycost, int64_t lo_len,
                 const int* d_datekey, const int* d_year, int d_len, const int* p_partkey,
                 const int* p_mfgr, int p_len, const int* s_suppkey, const int* s_region, int s_len,
                 const int* c_custkey, const int* c_region, const int* c_nation, int c_len,
                 int d_val_len, int c_region_eq, int s_region_eq, int mfgr_a, int mfgr_b, int* res,
                 int nthreads);

/* src/gpudb/CPUProcessing.cu:1786-1819 merge: fold resGPU into resCPU (int[6*n] layout). */
void orc_merge(int* res_cpu, const int* res_gpu, int num_groups);

#ifdef __cplusplus
}
#endif

#endif
