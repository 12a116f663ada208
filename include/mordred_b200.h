/*
 * mordred_b200.h — C ABI of the B200 (sm_100a) star-query hot path.
 *
 * Every entry point takes plain device pointers and sizes, is stream-ordered and
 * asynchronous on the stream it is given (NULL = legacy default stream), never
 * allocates on the query path and returns an int status (MB_OK = 0). Kernels report
 * data errors (a key outside its hash table, a group index outside the result array,
 * a pipeline wait that ran out) through a per-device status word that
 * mb_device_status() reads; they never trap.
 *
 * Ownership follows the reference: the caller allocates and zeroes every hash table
 * and result buffer (src/gpudb/QueryOptimizer.cu:2726-2748,3554-3571,
 * src/ssb/q21.cu:151-166); kernels accumulate into what they are given, so several
 * calls (segment groups, CPU + GPU halves) can add into one result.
 *
 * Each entry point names the reference interface it replaces (file:line within the
 * reference project).
 */
#ifndef MORDRED_B200_H
#define MORDRED_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A cudaStream_t passed as an opaque pointer (NULL = legacy default stream). */
typedef void* mb_stream_t;

/* ---- status codes ------------------------------------------------------------ */
#define MB_OK 0
#define MB_ERR_ARG 1         /* bad argument (NULL where required, bad enum, bad size) */
#define MB_ERR_ALIGN 2       /* a column or table pointer breaks the required alignment */
#define MB_ERR_LAUNCH 3      /* kernel launch failed */
#define MB_ERR_CUDA 4        /* a CUDA runtime call failed */
#define MB_ERR_NODEV 5       /* no CUDA device / device init failed */
#define MB_ERR_SIZE 6        /* size beyond a documented maximum */

/* ---- device status bits (sticky until cleared by mb_device_status) ----------- */
#define MB_STATUS_PROBE_RANGE 0x1u  /* (key - key_min) % num_slots < 0: row treated as a miss */
#define MB_STATUS_GROUP_RANGE 0x2u  /* group index outside [0, total_val): row skipped */
#define MB_STATUS_TIMEOUT 0x4u      /* a bounded pipeline wait ran out; result incomplete */
#define MB_STATUS_OVERFLOW 0x8u     /* an offset list was full: rows past its capacity were counted, not written */

/* ---- enums ---------------------------------------------------------------------- */
/* Filter modes: KernelArgs.h:44-86 (pred_eq, pred_between, pred_eq_or_eq),
 * build mode numbering GPUProcessing.h:971-982 (0 = EQ, 1 = BETWEEN, 2 = EQ OR EQ). */
#define MB_FILTER_EQ 0
#define MB_FILTER_BETWEEN 1
#define MB_FILTER_EQ_OR_EQ 2

/* Hash-table layouts. slot = (key - key_min) % num_slots (crystal/join.cuh:3).
 *  MB_HT_KEY      int ht[num_slots]; ht[slot] = key; nonzero = present; no payload
 *                 (BlockBuildSelectivePHT_1 / BlockProbeAndPHT_1, crystal/join.cuh:5-82,167-234)
 *  MB_HT_KEY_VAL  int ht[2*num_slots]; {key, val}; the 8-byte slot nonzero = present;
 *                 payload = upper 32 bits = val (crystal/join.cuh:84-165,236-311)
 *  MB_HT_VAL_OFF  int ht[2*num_slots]; {val, row+1}; the 8-byte slot nonzero = present;
 *                 payload = lower 32 bits = val (engine layout, BlockLibrary.cuh:86-111,594-735) */
#define MB_HT_KEY 0
#define MB_HT_KEY_VAL 1
#define MB_HT_VAL_OFF 2
/* No table: the probe passes through the group value an earlier join found. fkey is an
 * int list of dimension rows read at the call's row position k (an offset list's dim_off
 * array, or indexed by row when the call has no list), ht is the dimension column (or its
 * per-segment cache-slot array under segment addressing) read at that dimension row, and
 * num_slots the dimension's rows (a row outside [0, num_slots) sets
 * MB_STATUS_PROBE_RANGE and is dropped). Every row is present.
 * (BlockReadFilteredOffset, src/gpudb/BlockLibrary.cuh:484-541; GPUProcessing.h:198-205) */
#define MB_HT_PASS 3

/* Aggregates (int32 arithmetic, then widened to 64 bits, as q11.cu:74, q41.cu:76). */
#define MB_AGG_SUM 0   /* a0           */
#define MB_AGG_SUB 1   /* a0 - a1      (KernelArgs.h:20-24, group-by kernels) */
#define MB_AGG_MUL 2   /* a0 * a1      (KernelArgs.h:26-30, aggregate kernels) */
#define MB_AGG_MUL_PAYLOAD 3 /* a0 * payload of probe 0 (src/ops/join.cu:73) */

/* Result layouts. */
#define MB_RES_SCALAR 0   /* unsigned long long res[1] */
#define MB_RES_ENGINE6 1  /* int res[6*total_val]: g1..g4 at [6h..6h+3], u64 sum at [6h+4] (GPUProcessing.h:143-150) */
#define MB_RES_CRYSTAL4 2 /* int res[4*total_val]: two keys at [4h],[4h+1], u64 sum at [4h+2] (q21.cu:65-68) */
#define MB_RES_DENSE 3    /* unsigned long long res[total_val] (sums only) */

#define MB_MAX_FILTERS 3
#define MB_MAX_PROBES 4

/* ---- generic fused star query ------------------------------------------------- */
typedef struct mb_filter {
  const int* col;  /* fact column (or per-segment cache-slot index array in segment mode) */
  int mode;        /* MB_FILTER_* */
  int c1, c2;      /* EQ: x == c1; BETWEEN: c1 <= x <= c2; EQ_OR_EQ: x == c1 || x == c2 */
} mb_filter;

typedef struct mb_probe {
  const int* fkey;          /* fact foreign-key column (or cache-slot index array) */
  const int* ht;            /* hash table in `layout` */
  int num_slots;            /* ht_len */
  int key_min;              /* keys_min */
  int layout;               /* MB_HT_* */
  int min_val;              /* group term (payload - min_val) * unique_val */
  int unique_val;
  int res_slot;             /* ENGINE6: key column 0..3; CRYSTAL4: 0 or 1; -1: payload not stored */
  const uint32_t* presence; /* optional presence bitmap built by mb_build_* (bit s = slot s present) */
} mb_probe;

typedef struct mb_star_args {
  int64_t num_rows;
  int num_filters;
  mb_filter filter[MB_MAX_FILTERS];
  int num_probes;           /* probes run in array order */
  mb_probe probe[MB_MAX_PROBES];
  const int* aggr[2];       /* aggregate columns (aggr[1] NULL for MB_AGG_SUM) */
  int agg_op;               /* MB_AGG_* */
  int total_val;            /* number of groups (1 for MB_RES_SCALAR) */
  int group_bias;           /* constant added to the group sum before % total_val */
  int res_layout;           /* MB_RES_* */
  void* res;                /* device result, zeroed by the caller; accumulated into */
  unsigned long long* count;/* optional: rows passing the first count_after filters (u64, accumulated) */
  int count_after;          /* -1 = rows passing every filter and probe */
  /* Segment-cache addressing (src/gpudb/GPUProcessing.h:54-67). When gpu_cache is
   * non-NULL every column field above holds a per-segment cache-slot index array and
   * row r of the call reads gpu_cache[slot(seg(r)) * segment_size + r % segment_size]. */
  const int* gpu_cache;
  const short* segment_group; /* virtual segment -> segment id; NULL: (start_offset + r) / segment_size */
  int64_t start_offset;
  int segment_size;           /* power of two (reference: 1,048,576) */
  /* launch configuration; 0 = the tuned default for this shape */
  int threads;                /* consumer threads per CTA: 128, 256 or 512 (plus one producer warp);
                               * 640 or 768 (20 or 24 warps sharing 16 tile slices, 8 rows a
                               * thread) where the query shape has such a variant, else 512 */
  int items_per_thread;       /* fact rows per consumer thread per tile: 4, 8 or 16 */
  int stages;                 /* 2..8 bulk-copy stages */
  int grid;                   /* CTAs; 0 = one wave of resident CTAs */
  int group_mode;             /* 0 auto, 1 groups in shared memory (flushed per CTA), 2 global atomics per row */
  /* Offset-list input (optional): rows[k], k < num_rows, is the physical fact row the call
   * visits at position k (an offset list from mb_star_select, or from the CPU). Columns are
   * read at rows[k] (under segment addressing through the slot of segment rows[k] >>
   * log2(segment_size); segment_group and start_offset are then unused). The GPU3 forms of
   * the engine kernels (src/gpudb/GPUProcessing.h:157-273, 393-494, 1385-1524, 1610-1846).
   * The launch fields above are ignored for a list. */
  const int* rows;
  /* Cluster-resident mirrors of the sparse phase's hash tables (a presence bit, or a 4-bit
   * payload code, per slot, spread over the shared memory of a cluster of CTAs, so those
   * probes read on-chip memory instead of L2): 0 = the tuned default for the shape (large
   * calls only), 1 = never, 2 = whenever the tables fit. Results are the same either way. */
  int mirrors;
  /* Second sparse round packed across the warp (the rows the first selective table probe
   * kept are moved one a lane before the later probes and the aggregate run): 0 = the
   * tuned default for the shape, 1 = never, 2 = where the shape has a packed variant,
   * 3 = packed, with each tile's stage handed back to the bulk-copy producer before its
   * last batch of survivors is probed (their columns held in registers), 4 = unpacked,
   * with that early return. Results are the same either way. */
  int pack;
} mb_star_args;

/* Fused filter -> chained probe -> group-by/aggregate over the fact table.
 * Generalises filter_probe_group_by_GPU2 / probe_group_by_GPU2 / filter_probe_aggr_GPU2 /
 * probe_aggr_GPU2 (src/gpudb/GPUProcessing.h:17-155,275-391,1526-1776) and the SSB
 * probe kernels (src/ssb/q11.cu:25-93, q21.cu:25-72, q41.cu:25-80). */
int mb_star_query(const mb_star_args* args, mb_stream_t stream);

/* ---- Crystal-level builds and the src/ops operators ----------------------------- */
/* Filtered perfect-hash build. filter_col NULL = no filter. dim_val NULL builds the
 * MB_HT_KEY layout (BlockBuildSelectivePHT_1), else MB_HT_KEY_VAL (…_PHT_2).
 * presence (optional, zeroed by the caller, (num_slots+31)/32 words) receives the slot bitmap.
 * Replaces build_hashtable_s/p/c/d (src/ssb/q21.cu:74-138, src/ssb/q41.cu:82-167). */
int mb_build_pht(const int* filter_col, int filter_mode, int c1, int c2,
                 const int* dim_key, const int* dim_val, int num_tuples,
                 int* ht, int num_slots, int key_min, uint32_t* presence,
                 mb_stream_t stream);

/* Unfiltered PHT_2 build: src/ops/join.cu:21-40 build_kernel. */
int mb_join_build(const int* dim_key, const int* dim_val, int num_tuples,
                  int* hash_table, int num_slots, mb_stream_t stream);

/* Probe and sum fact_val * dim_val: src/ops/join.cu:42-85 probe_kernel. */
int mb_join_probe(const int* fact_fkey, const int* fact_val, int num_tuples,
                  const int* hash_table, int num_slots, unsigned long long* res,
                  mb_stream_t stream);

/* ---- SSB query kernels with the reference signatures ---------------------------- */
/* src/ssb/q11.cu:25-93 QueryKernel: revenue += sum(extendedprice*discount) over
 * 1<=discount<=3, quantity<25, 19930000<orderdate<19940000; d_total (optional) +=
 * rows passing the discount and quantity predicates. */
int mb_q11_query(const int* lo_orderdate, const int* lo_discount, const int* lo_quantity,
                 const int* lo_extendedprice, int lo_num_entries,
                 unsigned long long* revenue, int* d_total, mb_stream_t stream);

/* src/ssb/q21.cu:25-72 probe: res int[4*7000], group (brand*7 + year-1992) % 7000. */
int mb_q21_probe(const int* lo_orderdate, const int* lo_partkey, const int* lo_suppkey,
                 const int* lo_revenue, int lo_len,
                 const int* ht_s, int s_len, const int* ht_p, int p_len,
                 const int* ht_d, int d_len, int* res, mb_stream_t stream);

/* src/ssb/q41.cu:25-80 probe: res int[4*175], group (c_nation*7 + year-1992) % 175. */
int mb_q41_probe(const int* lo_orderdate, const int* lo_partkey, const int* lo_custkey,
                 const int* lo_suppkey, const int* lo_revenue, const int* lo_supplycost,
                 int lo_len, const int* ht_p, int p_len, const int* ht_s, int s_len,
                 const int* ht_c, int c_len, const int* ht_d, int d_len, int* res,
                 mb_stream_t stream);

/* The Query B probe of mb_q41_probe (same arguments, same result) for callers that
 * cannot let a library allocate device memory — an executor that sizes every device
 * buffer in its own arena up front, or a thread that must not take cudaMalloc's
 * device-wide synchronisation. It has no counterpart in the reference. Its scratch (the
 * status word and the supplier table's presence bitmap) is a fixed 33,024-byte array in
 * the library's device image, present on every device that loads the library until
 * the process exits; nothing is allocated. The first call on a device sets up (device
 * limits, kernel attributes, the array's device address) with that device current;
 * make that first call before any stream capture. s_len above 262,144 returns
 * MB_ERR_SIZE. Every call reuses the one array: the status word is cleared at the start
 * of each call, and calls whose work overlaps on the GPU (other streams, other host
 * threads) race on it — serialise them. status (optional, device word) receives the
 * call's MB_STATUS_* bits. */
int mb_q41_probe_noalloc(const int* lo_orderdate, const int* lo_partkey, const int* lo_custkey,
                         const int* lo_suppkey, const int* lo_revenue, const int* lo_supplycost,
                         int lo_len, const int* ht_p, int p_len, const int* ht_s, int s_len,
                         const int* ht_c, int c_len, const int* ht_d, int d_len, int* res,
                         unsigned int* status, mb_stream_t stream);

/* ---- engine (src/gpudb) kernel arguments, restated as plain C ------------------- */
/* KernelArgs.h:270-286 filterArgsGPU; device predicate function pointers become mode1/mode2. */
typedef struct mb_filterArgsGPU {
  const int* filter_idx1;
  const int* filter_idx2;
  int compare1, compare2, compare3, compare4;
  int mode1, mode2;
} mb_filterArgsGPU;

/* KernelArgs.h:146-169 probeArgsGPU (slot 1..4 = supplier, customer, part, date). */
typedef struct mb_probeArgsGPU {
  const int* key_idx1; const int* key_idx2; const int* key_idx3; const int* key_idx4;
  const int* ht1; const int* ht2; const int* ht3; const int* ht4;
  int dim_len1, dim_len2, dim_len3, dim_len4;
  int min_key1, min_key2, min_key3, min_key4;
} mb_probeArgsGPU;

/* KernelArgs.h:218-242 groupbyArgsGPU; the device group function pointer becomes mode
 * (0 = aggr1 - aggr2, 1 = aggr1 * aggr2). */
typedef struct mb_groupbyArgsGPU {
  const int* aggr_idx1; const int* aggr_idx2;
  const int* group_idx1; const int* group_idx2; const int* group_idx3; const int* group_idx4;
  int min_val1, min_val2, min_val3, min_val4;
  int unique_val1, unique_val2, unique_val3, unique_val4;
  int total_val;
  int mode;
} mb_groupbyArgsGPU;

/* KernelArgs.h:196-205 buildArgsGPU. */
typedef struct mb_buildArgsGPU {
  const int* key_idx;
  const int* val_idx;
  int num_slots;
  int val_min;
  int val_max;
} mb_buildArgsGPU;

/* GPUProcessing.h:17-155 filter_probe_group_by_GPU2, launched by
 * CPUGPUProcessing.cu:221-354 call_pfilter_probe_group_by_GPU. res = int[6*total_val]. */
int mb_filter_probe_group_by_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs,
                                  const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs,
                                  int num_tuples, int* res, int start_offset,
                                  const short* segment_group, mb_stream_t stream);

/* GPUProcessing.h:275-391 probe_group_by_GPU2 (CPUGPUProcessing.cu:802-916). */
int mb_probe_group_by_GPU2(const int* gpuCache, const mb_probeArgsGPU* pargs,
                           const mb_groupbyArgsGPU* gargs, int num_tuples, int* res,
                           int start_offset, const short* segment_group, mb_stream_t stream);

/* GPUProcessing.h:1675-1776 filter_probe_aggr_GPU2: u64 sum of aggr1*aggr2 at res[4]. */
int mb_filter_probe_aggr_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs,
                              const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs,
                              int num_tuples, int* res, int start_offset,
                              const short* segment_group, mb_stream_t stream);

/* GPUProcessing.h:927-997 build_GPU2: engine layout {val, row+1}. */
int mb_build_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs,
                  const mb_buildArgsGPU* bargs, int num_tuples, int* hash_table,
                  int start_offset, const short* segment_group, mb_stream_t stream);

/* KernelArgs.h:306-315 offsetGPU (declared here for the offset-list forms below): a list of
 * physical fact rows and, per dimension slot 1..4 (supplier, customer, part, date), the
 * dimension row each fact row joined with. */
typedef struct mb_offsetGPU {
  int* lo_off;
  int* dim_off1; int* dim_off2; int* dim_off3; int* dim_off4;
} mb_offsetGPU;

/* ---- offset-list (GPU3) forms and the remaining engine kernels --------------------
 * The list forms visit the num_tuples physical fact rows of offset->lo_off. For a
 * dimension slot with both key_idx and ht set the row probes that (VAL_OFF) table; for a
 * slot with only gargs->group_idx set the group value is gpuCache's dimension column
 * group_idx read at the row's offset->dim_off entry (an earlier join's match, which the
 * caller guarantees is a row of that dimension); other slots contribute group value 0.
 * Group-by forms: res = int[6*total_val], sum of aggr1 - aggr2 (gargs->mode 1: aggr1 *
 * aggr2); aggregate forms: u64 sum of aggr1 * aggr2 at res[4]. */
/* GPUProcessing.h:157-273 filter_probe_group_by_GPU3 (filters BETWEEN compare1..2, 3..4). */
int mb_filter_probe_group_by_GPU3(const int* gpuCache, const mb_offsetGPU* offset,
                                  const mb_filterArgsGPU* fargs, const mb_probeArgsGPU* pargs,
                                  const mb_groupbyArgsGPU* gargs, int num_tuples, int* res,
                                  mb_stream_t stream);
/* GPUProcessing.h:393-494 probe_group_by_GPU3. */
int mb_probe_group_by_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_probeArgsGPU* pargs,
                           const mb_groupbyArgsGPU* gargs, int num_tuples, int* res, mb_stream_t stream);
/* GPUProcessing.h:1385-1470 groupByGPU: no probes; every listed row is grouped by the
 * passed-through group values. */
int mb_groupByGPU(const int* gpuCache, const mb_offsetGPU* offset, const mb_groupbyArgsGPU* gargs,
                  int num_tuples, int* res, mb_stream_t stream);
/* GPUProcessing.h:1472-1524 aggregationGPU: u64 sum of aggr1 * aggr2 over lo_off at res[4]
 * (a missing aggregate column reads as 0, as BlockSetValue, so nothing is added). */
int mb_aggregationGPU(const int* gpuCache, const int* lo_off, const mb_groupbyArgsGPU* gargs,
                      int num_tuples, int* res, mb_stream_t stream);
/* GPUProcessing.h:1526-1608 probe_aggr_GPU2: the date probe (slot 4) only, then the
 * aggregate, over a segment range. */
int mb_probe_aggr_GPU2(const int* gpuCache, const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs,
                       int num_tuples, int* res, int start_offset, const short* segment_group,
                       mb_stream_t stream);
/* GPUProcessing.h:1610-1673 probe_aggr_GPU3: probe_aggr_GPU2 over an offset list. */
int mb_probe_aggr_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_probeArgsGPU* pargs,
                       const mb_groupbyArgsGPU* gargs, int num_tuples, int* res, mb_stream_t stream);
/* GPUProcessing.h:1778-1846 filter_probe_aggr_GPU3: the second filter (compare3..4) only —
 * the first ran where the list was made — then the date probe and the aggregate. */
int mb_filter_probe_aggr_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_filterArgsGPU* fargs,
                              const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs, int num_tuples,
                              int* res, mb_stream_t stream);
/* GPUProcessing.h:999-1028 build_GPU3: the engine build over the dimension rows listed in
 * dim_off (row id = the listed row); no filter (fargs->filter_idx1 must be NULL). */
int mb_build_GPU3(const int* gpuCache, const int* dim_off, const mb_filterArgsGPU* fargs,
                  const mb_buildArgsGPU* bargs, int num_tuples, int* hash_table, mb_stream_t stream);
/* GPUProcessing.h:1030-1113 build_GPU_minmax: build_GPU2 that also folds the smallest and
 * largest key of the rows passing the filter into *min_global / *max_global (device ints,
 * initialised by the caller; each CTA starts from bargs->val_max / val_min as the
 * reference's blocks do). */
int mb_build_GPU_minmax(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_buildArgsGPU* bargs,
                        int num_tuples, int* hash_table, int* min_global, int* max_global, int start_offset,
                        const short* segment_group, mb_stream_t stream);
/* GPUProcessing.h:1115-1172 build_GPU_minmax2: build_GPU3 with the key range. */
int mb_build_GPU_minmax2(const int* gpuCache, const int* dim_off, const mb_filterArgsGPU* fargs,
                         const mb_buildArgsGPU* bargs, int num_tuples, int* hash_table, int* min_global,
                         int* max_global, mb_stream_t stream);

/* ---- batched multi-query execution ------------------------------------------------ */
/* Many star queries over one resident fact table in one launch: every fact tile is
 * loaded once, each dimension is read once per row through a packed attribute table
 * (PAT: one 32-bit word per hash slot holding the dimension row's attributes, bit 31 =
 * row present), and every query of the batch evaluates its range predicates and
 * aggregate on that shared row. Each query's result equals running it alone through
 * mb_star_query with per-query filtered hash tables (the reference runs one query at a
 * time: src/gpudb/QueryProcessing.cu:1347-1471). No counterpart kernel exists in the
 * reference. */
#define MB_BATCH_MAX_QUERIES 256
#define MB_BATCH_MAX_PREDS 4

/* Row schema: fact columns 0..8, then the four dimension words. */
#define MB_COL_ORDERDATE 0
#define MB_COL_QUANTITY 1
#define MB_COL_DISCOUNT 2
#define MB_COL_EXTENDEDPRICE 3
#define MB_COL_SUPPKEY 4
#define MB_COL_CUSTKEY 5
#define MB_COL_PARTKEY 6
#define MB_COL_REVENUE 7
#define MB_COL_SUPPLYCOST 8
#define MB_COL_DIM_S 9   /* supplier word, looked up by suppkey */
#define MB_COL_DIM_C 10  /* customer word, by custkey */
#define MB_COL_DIM_P 11  /* part word, by partkey */
#define MB_COL_DIM_D 12  /* date word, by orderdate */
#define MB_NUM_FACT_COLS 9
/* A field: `width` bits at `shift` of column `col` (width 32 = the whole signed value). */
#define MB_FIELD(col, shift, width) (((col) << 11) | ((shift) << 6) | (width))

typedef struct mb_pat {
  const unsigned int* words;  /* words[(key - key_min) % slots] */
  int slots, key_min;
} mb_pat;

typedef struct mb_batch_query {
  int num_preds;                          /* lo <= field <= hi, all must hold */
  int pred_field[MB_BATCH_MAX_PREDS];
  int pred_lo[MB_BATCH_MAX_PREDS], pred_hi[MB_BATCH_MAX_PREDS];
  int dims_required;                      /* bit d: the row's dimension d (S,C,P,D) must exist */
  int agg_op;                             /* MB_AGG_SUM / SUB / MUL over agg_field[0..1] */
  int agg_field[2];
  int num_keys;                           /* group index = sum (key - key_min) * key_mul % total_val */
  int key_field[2], key_min[2], key_mul[2];
  int total_val;
  int res_layout;                         /* MB_RES_SCALAR, MB_RES_CRYSTAL4 (keys 0,1 stored) or MB_RES_DENSE */
  void* res;                              /* zeroed by the caller; accumulated into */
} mb_batch_query;

typedef struct mb_batch_args {
  int64_t num_rows;
  const int* fact[MB_NUM_FACT_COLS];      /* device columns by MB_COL_* (NULL where unused) */
  mb_pat dim[4];                          /* S, C, P, D */
  int num_queries;                        /* 1 .. MB_BATCH_MAX_QUERIES */
  const mb_batch_query* queries;          /* host array, copied into the launch */
  void* workspace;                        /* device, >= mb_batch_workspace_bytes(), 16-byte aligned */
  size_t workspace_bytes;
  /* consumer threads x rows per thread per stage: 256x4, 512x4, 512x2, 768x1, 768x2 or
   * 960x1 (0 = default 768x1); stages 2..8 (0 = 2); grid 0 = one CTA per SM */
  int threads, items_per_thread, stages, grid;
  int smem_group_bytes;                   /* shared memory for small group arrays; -1 default, 0 none */
  /* Segment-cache addressing (optional; src/gpudb/GPUProcessing.h:54-67 for one query):
   * when gpu_cache is non-NULL, fact[c] is column c's per-segment cache-slot array and row r
   * of the batch reads gpu_cache[slot * segment_size + r % segment_size], slot =
   * fact[c][segment_group[r / segment_size]] (r / segment_size without a list). One launch
   * thus scans a list of cached or staged segments for every query of the batch. */
  const int* gpu_cache;
  const short* segment_group;
  int segment_size;                       /* power of two */
} mb_batch_args;

/* Build a PAT: for each dimension row i, words[(key[i] - key_min) % slots] =
 * 0x80000000 | attr0 << shift0 | attr1 << shift1 | attr2 << shift2 for the fields
 * (MB_FIELD(.., shift, width)) given; attributes must fit their widths (else
 * MB_STATUS_GROUP_RANGE is set and the row is stored without them). words is zeroed by
 * the caller. */
int mb_pat_build(const int* dim_key, int num_rows, int key_min, int slots,
                 const int* attr0, int field0, const int* attr1, int field1,
                 const int* attr2, int field2, unsigned int* words, mb_stream_t stream);

/* Device workspace the batch needs: for every predicate attribute, a table mapping each
 * value of the queries' range hull to the bitmask of queries that accept it. */
size_t mb_batch_workspace_bytes(const mb_batch_args* args);

/* Run a batch of queries: one small kernel fills the workspace's query masks, then one
 * persistent kernel scans the fact table once. */
int mb_batch_run(const mb_batch_args* args, mb_stream_t stream);

/* ---- selection with compaction: offset lists for CPU/GPU handoff ---------------- */

/* Rows passing args' filters and probes (aggregation fields ignored) appended to an
 * offset list: lo_off[k] = physical row (start_offset + row, or the segment-mapped row
 * under segment addressing), dim_off[p][k] (optional per probe) = the probe's output:
 * VAL_OFF tables give the dimension row (ht[2h+1] - 1), KEY_VAL tables the payload, KEY
 * tables 0. *total (device int, zeroed by the caller) is the list cursor; entries past
 * `capacity` are counted but not written and set MB_STATUS_OVERFLOW. in_rows (optional,
 * device) restricts the pass to the listed physical rows (num_in of them). The order of
 * the list is not deterministic; its set of rows is. Restates filter_probe_GPU2/3,
 * probe_GPU2/3 and filter_GPU2/3 (src/gpudb/GPUProcessing.h:496-925, 1174-1383). */
int mb_star_select(const mb_star_args* args, const int* in_rows, int64_t num_in, int* lo_off,
                   int* const* dim_off, int64_t capacity, int* total, mb_stream_t stream);

/* The engine forms over the segment cache (SEGMENT_SIZE 1,048,576): column fields are
 * per-segment slot-index arrays into gpuCache; probes use engine (VAL_OFF) tables for
 * each dimension slot whose key_idx and ht are both set; out_off arrays hold
 * num_tuples entries. The GPU3 forms take the physical rows of in_off->lo_off and pass
 * in_off's dimension offsets through to slots they do not probe. */
int mb_filter_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_offsetGPU* out_off,
                   int num_tuples, int* total, int start_offset, const short* segment_group,
                   mb_stream_t stream);
int mb_filter_probe_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_probeArgsGPU* pargs,
                         const mb_offsetGPU* out_off, int num_tuples, int* total, int start_offset,
                         const short* segment_group, mb_stream_t stream);
int mb_probe_GPU2(const int* gpuCache, const mb_probeArgsGPU* pargs, const mb_offsetGPU* out_off,
                  int num_tuples, int* total, int start_offset, const short* segment_group,
                  mb_stream_t stream);
int mb_filter_GPU3(const int* gpuCache, const mb_offsetGPU* in_off, const mb_filterArgsGPU* fargs,
                   const mb_offsetGPU* out_off, int num_tuples, int* total, mb_stream_t stream);
int mb_filter_probe_GPU3(const int* gpuCache, const mb_offsetGPU* in_off, const mb_filterArgsGPU* fargs,
                         const mb_probeArgsGPU* pargs, const mb_offsetGPU* out_off, int num_tuples,
                         int* total, mb_stream_t stream);
int mb_probe_GPU3(const int* gpuCache, const mb_offsetGPU* in_off, const mb_probeArgsGPU* pargs,
                  const mb_offsetGPU* out_off, int num_tuples, int* total, mb_stream_t stream);

/* ---- learned planner: the cost MLP (no counterpart kernel in the reference, which
 * plans with the analytic model of src/gpudb/CostModel.cu:283-440) ------------------- */
/* 24 features -> 64 -> 64 -> 2 outputs (predicted log CPU ms, log GPU ms of a segment),
 * ReLU, fp32. params: W1[24][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2] (W[i][j]:
 * input i -> unit j), 5,890 floats. All pointers are device pointers. */
#define MB_MLP_IN 24
#define MB_MLP_HIDDEN 64
#define MB_MLP_OUT 2
#define MB_MLP_PARAMS 5890
/* y[batch][2] = MLP(x[batch][24]). */
int mb_mlp_forward(const float* params, const float* x, int batch, float* y, mb_stream_t stream);
/* grads[5890] += d/dparams of 1/(2*batch) * sum (MLP(x) - target)^2 (grads zeroed by the
 * caller); loss_sum (optional) += 1/2 * sum (MLP(x) - target)^2. Gradients are summed
 * with fp32 atomics, so their last bits vary between runs. */
int mb_mlp_backward(const float* params, const float* x, const float* target, int batch,
                    float* grads, float* loss_sum, mb_stream_t stream);
/* One Adam step on n parameters (an L2 term weight_decay * param is added to each
 * gradient first); step counts from 1. */
int mb_mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr,
                float beta1, float beta2, float eps, int step, float weight_decay,
                mb_stream_t stream);

/* ---- analytic cost model and segment placement (src/gpudb/CostModel.{h,cu}) ------- */
/* A fact pipeline for costing: filters, then probes, then (optionally) a group-by or
 * aggregate over num_aggr columns, with the fraction of rows each filter / probe keeps. */
typedef struct mb_cost_pipeline {
  int num_filters;
  double filter_sel[MB_MAX_FILTERS];
  int num_probes;
  double probe_sel[MB_MAX_PROBES];
  int group_by;   /* 1: a group-by / aggregate ends the pipeline */
  int num_aggr;   /* its aggregate columns (n_aggr_key) */
} mb_cost_pipeline;

/* CostModel.cu:283-363 calculate_cost for one placement: on_gpu[i] for the filters,
 * then the probes, then the group-by (1 = GPU). Returns ms (BW_CPU 42e6 and BW_PCI
 * 12e6 bytes per ms, CostModel.h:4-6) for `rows` rows, or -1 on bad arguments. */
double mb_cost_calculate(const mb_cost_pipeline* pipeline, const int* on_gpu, double rows);
/* The whole pipeline on the CPU. */
double mb_cost_cpu_ms(const mb_cost_pipeline* pipeline, double rows);
/* CostModel.cu:386-390 transfer_cost: `columns` int columns of `rows` rows over PCIe. */
double mb_cost_transfer_ms(double rows, int columns);
/* CostModel.cu:427-440 build_cost of a hash-table build over dim_rows rows on the CPU. */
double mb_cost_build_ms(double dim_rows);
/* Per-segment analytic estimates for one pipeline: cpu_ms[i] = the all-CPU cost of
 * rows[i] rows with the first filter's selectivity first_filter_sel[i] (optional);
 * gpu_ms[i] = the PCIe transfer of the segment's missing_cols[i] columns (optional, 0). */
int mb_cost_segments(const mb_cost_pipeline* pipeline, int n, const double* rows,
                     const double* first_filter_sel, const int* missing_cols,
                     double* cpu_ms, double* gpu_ms);
/* Split n segments between CPU and GPU (on_gpu[i] = 1: GPU) to minimise
 * max(cpu_fixed_ms + sum of CPU ms, gpu_fixed_ms + sum of GPU ms) — a device's fixed
 * cost counts only when it takes a segment — over a GPU/CPU time-ratio order;
 * *makespan_ms (optional) receives that maximum. No counterpart in the reference, which
 * places by segment residency (QueryOptimizer.cu:1674-1891). */
int mb_place_segments(int n, const double* cpu_ms, const double* gpu_ms, double cpu_fixed_ms,
                      double gpu_fixed_ms, unsigned char* on_gpu, double* makespan_ms);

/* ---- CPU operators (host columns; the CPU half of CPU/GPU split execution) ------- */
/* Host threads the CPU operators use at most (a persistent pool). */
int mb_cpu_threads(void);

/* Filtered perfect-hash build on the host: src/gpudb/CPUProcessing.cu:1034-1104
 * build_CPU, and the Crystal layouts of mb_build_pht. layout MB_HT_KEY (dim_val unused),
 * MB_HT_KEY_VAL {key, val} or MB_HT_VAL_OFF {val, row+1}. nthreads <= 0: all. Slots
 * out of range set MB_STATUS_PROBE_RANGE in *status (optional). */
int mb_cpu_build_pht(const int* filter_col, int filter_mode, int c1, int c2,
                     const int* dim_key, const int* dim_val, int num_tuples,
                     int* ht, int num_slots, int key_min, int layout, int nthreads,
                     unsigned int* status);

/* The fused star pipeline of mb_star_query over HOST columns and host hash tables
 * (CPUProcessing.cu:439-568, 723-866, 1628-1710). gpu_cache must be NULL; segment_size
 * > 0 maps virtual rows through segment_group as on the GPU, over plain host columns.
 * rows (optional) lists the virtual rows to process (an offset list from
 * mb_star_select); num_listed is its length. Results accumulate into args->res exactly
 * as the GPU path's do, so CPU and GPU partial results of one query merge by addition
 * (src/gpudb/CPUProcessing.cu:1786-1819 merge). Launch fields are ignored. */
int mb_cpu_star_query(const mb_star_args* args, const int* rows, int64_t num_listed,
                      int nthreads, unsigned int* status);

/* Selection with compaction on the host (filter_CPU / filter_probe_CPU / probe_CPU and their
 * list forms, src/gpudb/CPUProcessing.cu:3-437,1158-1333): the rows of the call (its
 * virtual rows, mapped through segment_group as in mb_cpu_star_query, or the listed ones)
 * passing a's filters and probes, written in row order: lo_off[k] = physical row,
 * dim_off[p][k] (optional per probe) = ht[2h+1] - 1 for VAL_OFF tables (the dimension
 * row), the payload for KEY_VAL, 0 for KEY. *total = rows passing; entries past capacity
 * are counted, not written, and set MB_STATUS_OVERFLOW in *status. The CPU half of a
 * query split CPU-select -> GPU-aggregate (the GPU3 forms above take the list). */
int mb_cpu_star_select(const mb_star_args* a, const int* rows, int64_t num_listed, int* lo_off,
                       int* const* dim_off, int64_t capacity, int64_t* total, int nthreads,
                       unsigned int* status);

/* ---- GPU segment cache (src/gpudb/CacheManager.{h,cu}) ---------------------------- */
/* Fact columns are split into segments of segment_size rows (reference SEGMENT_SIZE,
 * common.h:73). The cache owns one device pool of num_slots segment slots — the
 * kernels' gpuCache — and maps (column, segment) to a slot. mb_segcache_col_idx gives
 * a column's slot-per-segment array, the per-column index array of mb_star_query's
 * segment addressing. device < 0 keeps the pool in host memory (bookkeeping without a
 * GPU). Calls on one cache are serialised internally. */
#define MB_CACHE_LRU 0     /* admission evicts the least recently used segment */
#define MB_CACHE_LFU 1     /* ... the least frequently used */
#define MB_CACHE_WEIGHT 2  /* ... the one with the smallest benefit weight */

typedef struct mb_segcache mb_segcache;
typedef struct mb_segcache_stats {
  unsigned long long hits, misses;      /* mb_segcache_touch of resident / absent segments */
  unsigned long long admissions, evictions, bytes_h2d;
  unsigned long long resident;          /* slots in use */
} mb_segcache_stats;

/* NULL on bad arguments or when the pool cannot be allocated. num_segments <= 32767
 * (segment ids are 16-bit in segment_group lists, as the reference's short). */
mb_segcache* mb_segcache_create(int device, int64_t num_slots, int segment_size,
                                int num_columns, int num_segments, int policy);
void mb_segcache_destroy(mb_segcache* cache);
int* mb_segcache_pool(mb_segcache* cache);
/* Slot of (col, seg), -1 when not resident. */
int mb_segcache_slot(mb_segcache* cache, int col, int seg);
/* out[seg] = slot of (col, seg) or -1, for every segment (host array). */
int mb_segcache_col_idx(mb_segcache* cache, int col, int* out);
/* Start a query: segments it touches or admits from now on are pinned until the next
 * mb_segcache_begin_query. */
void mb_segcache_begin_query(mb_segcache* cache);
/* Record a use of (col, seg) by the running query (recency, frequency, hit/miss). */
int mb_segcache_touch(mb_segcache* cache, int col, int seg);
int mb_segcache_set_weight(mb_segcache* cache, int col, int seg, double weight);
/* Make (col, seg) resident, copying `rows` ints from host_src (pinned for asynchronous
 * copies) on `stream`; evicts by the cache's policy when no slot is free (never a
 * segment pinned by the running query: MB_ERR_SIZE when only those are left). */
int mb_segcache_admit(mb_segcache* cache, int col, int seg, const int* host_src, int rows,
                      mb_stream_t stream, int* slot_out);
/* Admit, in order, every listed column of every listed segment (a touch plus
 * mb_segcache_admit each). host_cols[col] is the host column, seg_rows[seg] the rows of
 * a segment. *done = segments whose columns are all resident; *copied (optional) +=
 * column segments copied. MB_ERR_SIZE when segment *done does not fit beside the
 * pinned segments (some of its columns may have been admitted). */
int mb_segcache_admit_segments(mb_segcache* cache, const int* cols, int ncols, const int* segs,
                               int nsegs, const int* const* host_cols, const int* seg_rows,
                               mb_stream_t stream, int* done, unsigned long long* copied);
int mb_segcache_evict(mb_segcache* cache, int col, int seg);
/* Epoch replacement (CacheManager.cu:534-588 SegmentReplacement): weights[col *
 * num_segments + seg] are benefit weights; the positive ones, heaviest first, are made
 * resident up to the slot count and every other resident segment is evicted.
 * host_cols[col] is the host column (NULL: never admitted), segment_rows[seg] the rows
 * of each segment. */
int mb_segcache_replace(mb_segcache* cache, const double* weights, const int* const* host_cols,
                        const int* segment_rows, mb_stream_t stream);
int mb_segcache_get_stats(mb_segcache* cache, mb_segcache_stats* out);
/* Take the nslots highest slots not yet reserved out of the cache's management (evicting
 * what they hold): admission and replacement never use them again, and the caller owns
 * them — a staging area for segments it streams through the pool without making them
 * resident (slot s at mb_segcache_pool() + s * segment_size). *first_slot = the lowest
 * reserved slot. MB_ERR_SIZE when no managed slot would be left. No counterpart in the
 * reference, whose executor admits every segment it reads. */
int mb_segcache_reserve(mb_segcache* cache, int64_t nslots, int64_t* first_slot);
/* Copy `rows` ints from host_src (pinned for an asynchronous copy) into reserved slot
 * `slot` on `stream`; the slot's map entry is the caller's to keep. MB_ERR_ARG for a slot
 * the cache manages. */
int mb_segcache_stage(mb_segcache* cache, int64_t slot, const int* host_src, int rows, mb_stream_t stream);

/* ---- synthetic data (seeded; identical on host and device) ---------------------- */
/* Fact column `col` (MB_LO_* in mordred_b200/csrc/ssbgen.h) rows [row0, row0+n) into a
 * device buffer. s_len/c_len/p_len give the foreign-key ranges. */
int mb_gen_fact_column(int col, uint64_t seed, int64_t row0, int64_t n,
                       int s_len, int c_len, int p_len, int* out, mb_stream_t stream);
/* Dimension column (MB_D_*, MB_S_*, MB_C_*, MB_P_*) rows [0, n) into a device buffer. */
int mb_gen_dim_column(int col, uint64_t seed, int64_t n, int* out, mb_stream_t stream);
/* Host versions (nthreads <= 0: all hardware threads). */
int mb_gen_fact_column_host(int col, uint64_t seed, int64_t row0, int64_t n,
                            int s_len, int c_len, int p_len, int* out, int nthreads);
int mb_gen_dim_column_host(int col, uint64_t seed, int64_t n, int* out, int nthreads);

/* ---- runtime ---------------------------------------------------------------------- */
int mb_version(void);
/* Per-device set-up (kernel attributes, the device status word). Called implicitly by
 * the first launch on a device; call it explicitly before capturing a CUDA graph. */
int mb_init(int device);
/* Read (and optionally clear) the device status bits; synchronises the device. */
int mb_device_status(int device, unsigned int* status, int clear);
const char* mb_error_string(int code);
/* Number of kernel launches issued by this library in this process (all devices). */
unsigned long long mb_launch_count(void);
/* 1 when the library's per-device state (the status word it cudaMalloc's and the kernel
 * attributes mb_init sets) exists on `device`, else 0. Touches no device and allocates
 * nothing: a caller can check that only allocation-free entry points ran. */
int mb_device_state_ready(int device);

#ifdef __cplusplus
}
#endif

#endif /* MORDRED_B200_H */
