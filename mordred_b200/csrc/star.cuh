// star.cuh — the fused star-query pipeline: its device-side plan and the host launcher.
//
// One persistent, warp-specialised kernel runs filter -> chained perfect-hash probes ->
// group-by / aggregate over the fact table:
//   * a producer warp streams fact-column tiles into shared memory with 1-D bulk copies
//     (cp.async.bulk, no multicast) into a ring of stages, each guarded by a "full"
//     mbarrier (transaction bytes) and an "empty" mbarrier (one arrival per consumer warp);
//   * each consumer warp owns a contiguous slice of every tile. A dense phase reads its
//     rows with 128-bit shared loads and applies the filters and the probes whose
//     presence bitmap sits in shared memory, keeping the selection as a bitmask; the
//     survivors are compacted (warp prefix sum) into a per-warp row list, and a sparse
//     phase runs the remaining L2-resident probes over that list with every lane busy,
//     issuing the table loads of all remaining probes at once (each probe's slot depends
//     only on the row's own key) before combining them in the reference's order;
//   * sums are 64-bit integers in registers (scalar), in a shared-memory group array
//     flushed with one 64-bit atomic per touched group per CTA, or 64-bit atomics in L2.
// The query shape (number of filters, of bitmap-decided probes and of table probes) is
// a template parameter for the common shapes, so their loops unroll to straight code;
// any other shape runs the same kernel with the counts read from the plan.
#pragma once

#include "common.cuh"

namespace mb {

constexpr int kMaxCols = MB_MAX_FILTERS + MB_MAX_PROBES + 2;
constexpr int kMaxStages = 8;
// A staged tile is cut into slices of 32 x items rows, one per consumer warp; launches with
// more than 16 consumer warps keep 16 slices a tile and hand the slices out round robin, so
// several warps probe earlier slices while others run the dense phase of later ones.
constexpr int kMaxTileSlices = 16;
__host__ __device__ constexpr int tile_slices(int consumer_warps) {
  return consumer_warps > kMaxTileSlices ? kMaxTileSlices : consumer_warps;
}
// Per-warp shared memory for the survivor list (a 16-bit row offset per slice row). The
// packed variants that return the stage early reuse it after the last batch's gather to
// hand the first probe's kept rows to their packed lanes: 32 rows of kXferWords ints (an
// odd stride, so the 32 rows fall in distinct banks).
constexpr int kXferWords = 7;
__host__ __device__ constexpr int star_list_bytes(int items, bool xfer) {
  return xfer && 32 * kXferWords * 4 > 64 * items ? 32 * kXferWords * 4 : 64 * items;
}
constexpr int kSmemGroupMax = 8192;            // groups kept in shared memory per CTA
constexpr int kBitmapSmemMaxBytes = 32768;     // largest presence bitmap staged (262,144 slots)
constexpr int kBitmapSmemTotalBytes = 40960;
constexpr int kBitmapDeriveMaxSlots8 = 65536;  // largest 8-byte-slot table whose bitmap a CTA derives
// Cluster-resident mirrors: narrow copies of the sparse phase's hash tables (1 presence bit
// or one 4-bit payload code per slot) spread over the shared memory of a thread-block
// cluster, each CTA holding a power-of-two share of at most this many 32-bit words.
constexpr int kMirrorMaxShareWords = 16384;   // 64 KB per CTA
constexpr int kMirrorMaxCluster = 8;           // portable cluster size
constexpr long long kMirrorMinRows = 8ll << 20;  // smaller calls do not repay building the mirrors
enum MirrorKind { kMirNone = 0, kMirBits = 1, kMirNibble = 2 };
// 4-bit payload codes: 0 absent, 1..14 present with payload min + code - 1, 15 present
// with a payload the code cannot hold (read the table itself).
constexpr unsigned kNibbleEscape = 15u;

enum GroupMode { kGroupScalar = 0, kGroupSmem = 1, kGroupGlobal = 2 };

struct StarPlan {
  long long n;       // rows in this call
  long long nfull;   // full tiles (the remainder runs with plain loads)
  int ncols;
  const int* col[kMaxCols];
  int nf;
  int f_col[MB_MAX_FILTERS], f_mode[MB_MAX_FILTERS], f_c1[MB_MAX_FILTERS], f_c2[MB_MAX_FILTERS];
  int np;
  int n_dense;                    // leading probes tested against a staged presence bitmap
  int sparse_p0;                  // first probe of the sparse phase: the leading bitmap-tested
                                  // probes whose payload is not needed stop before it, the
                                  // others are probed again there for their payload
  unsigned dense_bias;            // group terms (0 - min_val) * unique_val of probes < sparse_p0
  int sp_ord[MB_MAX_PROBES];      // tiled path: probe visited at sparse position q (the first
                                  // probe that can drop rows leads; the dense phase settled the
                                  // probes it passes, which are read only for their payloads)
  int p_col[MB_MAX_PROBES];
  const int* p_ht[MB_MAX_PROBES];
  int p_slots[MB_MAX_PROBES], p_kmin[MB_MAX_PROBES], p_layout[MB_MAX_PROBES];
  int p_min[MB_MAX_PROBES], p_mul[MB_MAX_PROBES], p_res_slot[MB_MAX_PROBES];
  const uint32_t* p_presence[MB_MAX_PROBES];
  int p_bm_off[MB_MAX_PROBES];    // byte offset of a staged bitmap in shared memory, -1 = none
  int p_bm_words[MB_MAX_PROBES];
  int a_col[2];
  int agg_op;
  int total_val, group_bias, res_layout;
  void* res;
  void* count;
  int count32;                    // count is an int* (q11's d_total) rather than u64*
  int count_after;
  int gmode;
  const int* gpu_cache;
  const short* seg_group;
  long long start_offset;
  int seg_shift;
  unsigned int* status;
  int stages;
  int smem_groups_off, smem_list_off, smem_stage_off, stage_bytes, smem_total;
  // cluster-resident mirrors (cluster > 1): probe p's mirror kind, its first word in the
  // cluster's word space, and the payload its codes count from; word w lives in CTA
  // w >> mir_shift at share word w & ((1 << mir_shift) - 1)
  int cluster;
  int mir_kind[MB_MAX_PROBES], mir_base[MB_MAX_PROBES], mir_words[MB_MAX_PROBES], mir_min[MB_MAX_PROBES];
  int mir_payload[MB_MAX_PROBES];  // 1: the probe's payload is read (from its code, else from the table)
  int mir_shift;
  int smem_mirror_off;
};

// Host: validate `a`, fill `plan`, pick the kernel variant and launch it on `stream`.
// count32 makes `count` an int* accumulator. `preset` supplies the device state (SM
// count, shared-memory limit, status word) instead of the library's own.
int launch_star(const mb_star_args* a, cudaStream_t stream, int count32, const DeviceState* preset = nullptr);

// Host: set per-device kernel attributes (dynamic shared memory opt-in).
int star_init_device(const DeviceState& ds);
// Host: the offset-list form of the pipeline (listq.cu): a->rows lists physical rows, or a
// probe passes a group value through (MB_HT_PASS). Arguments are validated here.
int launch_list(const mb_star_args* a, cudaStream_t stream, const DeviceState* ds);
int list_init_device(const DeviceState& ds);
// Host: the same for the batched multi-query kernel (batch.cu).
int batch_init_device(const DeviceState& ds);

}  // namespace mb
