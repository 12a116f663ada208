// star.cu — persistent, bulk-copy-staged fused star-query kernel (see star.cuh).
//
// Semantics follow the reference kernels row for row:
//   filters      GPUProcessing.h:74-86 (fact BETWEEN), crystal/pred.cuh (EQ, EQ OR EQ)
//   probes       crystal/join.cuh:5-165 (PHT_1 / PHT_2), BlockLibrary.cuh:86-111 (engine)
//   group index  GPUProcessing.h:143 ((g1-m1)*u1 + ... ) % total_val, int32 arithmetic
//   aggregate    q11.cu:74 (int32 product widened), GPUProcessing.h:149-150 (int32 difference)
// Rows are independent and every sum is a 64-bit integer, so the order in which tiles,
// rows and atomics are applied cannot change any result bit.
#include <algorithm>
#include <climits>
#include <cstring>

#include "star.cuh"

namespace mb {

__device__ __forceinline__ bool pass_filter(int x, int mode, int c1, int c2) {
  if (mode == MB_FILTER_BETWEEN) return x >= c1 && x <= c2;
  if (mode == MB_FILTER_EQ) return x == c1;
  return x == c1 || x == c2;
}

// Column pointer for the row `r` of this call (direct or through the segment cache).
__device__ __forceinline__ const int* row_ptr(const StarPlan& P, int c, long long r) {
  if (P.gpu_cache == nullptr) return P.col[c] + r;
  const long long vseg = r >> P.seg_shift;
  const int seg = P.seg_group ? static_cast<int>(P.seg_group[vseg])
                              : static_cast<int>((P.start_offset + r) >> P.seg_shift);
  const long long slot = P.col[c][seg];
  return P.gpu_cache + (slot << P.seg_shift) + (r & ((1ll << P.seg_shift) - 1));
}

// Loader over a tile staged in shared memory: thread t owns rows (j*THREADS + t)*4 + e.
template <int THREADS, int VPT>
struct SmemTileLoader {
  static constexpr int ITEMS = 4 * VPT;
  static constexpr int TILE = THREADS * ITEMS;
  const int* base;
  __device__ __forceinline__ void load(int c, int (&v)[ITEMS]) const {
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
      const int4 q = lds128(base + c * TILE + (j * THREADS + threadIdx.x) * 4);
      v[4 * j + 0] = q.x;
      v[4 * j + 1] = q.y;
      v[4 * j + 2] = q.z;
      v[4 * j + 3] = q.w;
    }
  }
};

// Loader for one remainder row read straight from global memory.
struct RowLoader {
  static constexpr int ITEMS = 1;
  const StarPlan* P;
  long long r;
  __device__ __forceinline__ void load(int c, int (&v)[1]) const { v[0] = __ldg(row_ptr(*P, c, r)); }
};

__device__ __forceinline__ void add_count(const StarPlan& P, unsigned long long& cnt, uint32_t sel) {
  cnt += static_cast<unsigned long long>(__popc(sel));
}

template <int ITEMS>
__device__ __forceinline__ void write_keys(const StarPlan& P, int h, const int (&gv)[MB_MAX_PROBES][ITEMS],
                                           int i) {
  int* res = static_cast<int*>(P.res);
  if (P.res_layout == MB_RES_ENGINE6) {
#pragma unroll
    for (int p = 0; p < MB_MAX_PROBES; ++p)
      if (p < P.np && P.p_res_slot[p] >= 0) res[6 * h + P.p_res_slot[p]] = gv[p][i];
  } else if (P.res_layout == MB_RES_CRYSTAL4) {
#pragma unroll
    for (int p = 0; p < MB_MAX_PROBES; ++p)
      if (p < P.np && P.p_res_slot[p] >= 0) res[4 * h + P.p_res_slot[p]] = gv[p][i];
  }
}

__device__ __forceinline__ unsigned long long* group_sum_ptr(const StarPlan& P, int h) {
  if (P.res_layout == MB_RES_ENGINE6)
    return reinterpret_cast<unsigned long long*>(static_cast<int*>(P.res) + 6 * h + 4);
  if (P.res_layout == MB_RES_CRYSTAL4)
    return reinterpret_cast<unsigned long long*>(static_cast<int*>(P.res) + 4 * h + 2);
  return static_cast<unsigned long long*>(P.res) + h;
}

// The per-row pipeline for the ITEMS rows a thread holds; `sel` marks valid rows.
template <class L>
__device__ __forceinline__ void process_rows(const StarPlan& P, const L& ld, uint32_t sel,
                                             unsigned long long& acc, unsigned long long& cnt,
                                             unsigned long long* s_sum, uint32_t* s_touch,
                                             const unsigned char* smem, bool& bad_probe,
                                             bool& bad_group) {
  constexpr int ITEMS = L::ITEMS;
  int v[ITEMS];

  // ---- filters (AND of all) --------------------------------------------------
#pragma unroll
  for (int f = 0; f < MB_MAX_FILTERS; ++f) {
    if (f >= P.nf) break;
    if (P.count_after == f) add_count(P, cnt, sel);
    if (sel == 0) break;
    ld.load(P.f_col[f], v);
    const int mode = P.f_mode[f], c1 = P.f_c1[f], c2 = P.f_c2[f];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i)
      if (!pass_filter(v[i], mode, c1, c2)) sel &= ~(1u << i);
  }
  if (P.count_after >= P.nf) add_count(P, cnt, sel);

  // ---- chained probes ----------------------------------------------------------
  int gv[MB_MAX_PROBES][ITEMS];
#pragma unroll
  for (int p = 0; p < MB_MAX_PROBES; ++p) {
    if (p >= P.np || sel == 0) break;
    ld.load(P.p_col[p], v);
    const int slots = P.p_slots[p], kmin = P.p_kmin[p], layout = P.p_layout[p];
    const int* ht = P.p_ht[p];
    const uint32_t* bm =
        P.p_bm_off[p] >= 0 ? reinterpret_cast<const uint32_t*>(smem + P.p_bm_off[p]) : nullptr;
    unsigned long long sv[ITEMS];
    // pass 1: compute slots and issue every table load before any is used
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      sv[i] = 0;
      if (sel & (1u << i)) {
        const int d = v[i] - kmin;
        const int h = (d >= 0 && d < slots) ? d : d % slots;
        if (h < 0) {
          sel &= ~(1u << i);
          bad_probe = true;
        } else if (bm != nullptr && !((bm[h >> 5] >> (h & 31)) & 1u)) {
          sel &= ~(1u << i);
        } else if (layout == MB_HT_KEY) {
          sv[i] = bm != nullptr ? 1ull : static_cast<unsigned long long>(static_cast<unsigned>(__ldg(ht + h)));
        } else {
          sv[i] = ldg_u64(ht + 2 * static_cast<long long>(h));
        }
      }
    }
    // pass 2: presence and payload
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (sel & (1u << i)) {
        if (sv[i] == 0) {
          sel &= ~(1u << i);
        } else {
          gv[p][i] = layout == MB_HT_KEY_VAL ? static_cast<int>(sv[i] >> 32)
                     : layout == MB_HT_VAL_OFF ? static_cast<int>(static_cast<unsigned>(sv[i]))
                                               : 0;
        }
      }
    }
  }
  if (P.count_after < 0) add_count(P, cnt, sel);
  if (sel == 0) return;

  // ---- aggregate -----------------------------------------------------------------
  int a0[ITEMS], a1[ITEMS];
  ld.load(P.a_col[0], a0);
  if (P.agg_op == MB_AGG_SUB || P.agg_op == MB_AGG_MUL) ld.load(P.a_col[1], a1);
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    if (!(sel & (1u << i))) continue;
    int val;
    if (P.agg_op == MB_AGG_SUM)
      val = a0[i];
    else if (P.agg_op == MB_AGG_SUB)
      val = static_cast<int>(static_cast<unsigned>(a0[i]) - static_cast<unsigned>(a1[i]));
    else if (P.agg_op == MB_AGG_MUL_PAYLOAD)
      val = static_cast<int>(static_cast<unsigned>(a0[i]) * static_cast<unsigned>(gv[0][i]));
    else
      val = static_cast<int>(static_cast<unsigned>(a0[i]) * static_cast<unsigned>(a1[i]));
    const unsigned long long w = static_cast<unsigned long long>(static_cast<long long>(val));
    if (P.gmode == kGroupScalar) {
      acc += w;
      continue;
    }
    unsigned hh = static_cast<unsigned>(P.group_bias);
#pragma unroll
    for (int p = 0; p < MB_MAX_PROBES; ++p)
      if (p < P.np)
        hh += static_cast<unsigned>(gv[p][i] - P.p_min[p]) * static_cast<unsigned>(P.p_mul[p]);
    const int h = static_cast<int>(hh) % P.total_val;
    if (h < 0) {
      bad_group = true;
      continue;
    }
    if (P.gmode == kGroupSmem) {
      atomicAdd(&s_sum[h], w);
      const uint32_t bit = 1u << (h & 31);
      if (!(s_touch[h >> 5] & bit)) {
        if (!(atomicOr(&s_touch[h >> 5], bit) & bit)) write_keys<ITEMS>(P, h, gv, i);
      }
    } else {
      write_keys<ITEMS>(P, h, gv, i);
      atomicAdd(group_sum_ptr(P, h), w);
    }
  }
}

template <int THREADS, int VPT>
__global__ void __launch_bounds__(THREADS, 1) star_kernel(const __grid_constant__ StarPlan P) {
  constexpr int ITEMS = 4 * VPT;
  constexpr int TILE = THREADS * ITEMS;
  constexpr int NWARPS = THREADS / 32;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long s_red[2 * NWARPS];

  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned long long* s_sum = reinterpret_cast<unsigned long long*>(smem + P.smem_groups_off);
  uint32_t* s_touch = reinterpret_cast<uint32_t*>(smem + P.smem_groups_off + 8 * P.total_val);
  int* stage_base = reinterpret_cast<int*>(smem + P.smem_stage_off);
  const int tid = threadIdx.x;
  const int stages = P.stages;

  // ---- set-up: group accumulators, staged presence bitmaps, barriers ----------
  if (P.gmode == kGroupSmem) {
    for (int g = tid; g < P.total_val; g += THREADS) s_sum[g] = 0;
    for (int w = tid; w < (P.total_val + 31) / 32; w += THREADS) s_touch[w] = 0;
  }
#pragma unroll
  for (int p = 0; p < MB_MAX_PROBES; ++p) {
    if (p >= P.np || P.p_bm_off[p] < 0) continue;
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + P.p_bm_off[p]);
    const int words = P.p_bm_words[p];
    if (P.p_presence[p] != nullptr) {
      for (int w = tid; w < words; w += THREADS) bm[w] = __ldg(P.p_presence[p] + w);
    } else {
      // derive presence from a MB_HT_KEY table: one warp ballot per 32 slots
      const int lane = tid & 31;
      for (int w = tid >> 5; w < words; w += NWARPS) {
        const int s = w * 32 + lane;
        const int k = s < P.p_slots[p] ? __ldg(P.p_ht[p] + s) : 0;
        const uint32_t b = __ballot_sync(0xffffffffu, k != 0);
        if (lane == 0) bm[w] = b;
      }
    }
  }
  if (tid == 0) {
    for (int s = 0; s < stages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  const long long G = gridDim.x;
  const long long b = blockIdx.x;
  const long long my_tiles = P.nfull > b ? (P.nfull - 1 - b) / G + 1 : 0;
  const uint32_t stage_words = static_cast<uint32_t>(P.ncols) * TILE;
  uint64_t policy = 0;
  if (tid == 0) policy = l2_policy_evict_first();

  auto issue = [&](long long k) {
    const int s = static_cast<int>(k % stages);
    const long long r0 = (b + k * G) * static_cast<long long>(TILE);
    int* dst = stage_base + s * stage_words;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bars[s], stage_words * 4u);
    if (P.gpu_cache == nullptr) {
      for (int c = 0; c < P.ncols; ++c) bulk_g2s(dst + c * TILE, P.col[c] + r0, TILE * 4, &bars[s], policy);
    } else {
      const long long vseg = r0 >> P.seg_shift;
      const int seg = P.seg_group ? static_cast<int>(P.seg_group[vseg])
                                  : static_cast<int>((P.start_offset + r0) >> P.seg_shift);
      const long long in_seg = r0 & ((1ll << P.seg_shift) - 1);
      for (int c = 0; c < P.ncols; ++c) {
        const long long slot = P.col[c][seg];
        bulk_g2s(dst + c * TILE, P.gpu_cache + (slot << P.seg_shift) + in_seg, TILE * 4, &bars[s], policy);
      }
    }
  };

  if (tid == 0) {
    const long long pre = my_tiles < stages ? my_tiles : stages;
    for (long long k = 0; k < pre; ++k) issue(k);
  }

  unsigned long long acc = 0, cnt = 0;
  bool bad_probe = false, bad_group = false;
  const uint32_t full = ITEMS == 32 ? 0xffffffffu : ((1u << ITEMS) - 1u);
  long long failed_at = -1;

  for (long long k = 0; k < my_tiles; ++k) {
    const int s = static_cast<int>(k % stages);
    const uint32_t parity = static_cast<uint32_t>((k / stages) & 1);
    const bool ok = mbar_wait_bounded(&bars[s], parity);
    if (ok) {
      SmemTileLoader<THREADS, VPT> ld{stage_base + s * stage_words};
      process_rows(P, ld, full, acc, cnt, s_sum, s_touch, smem, bad_probe, bad_group);
    }
    if (__syncthreads_or(!ok)) {
      failed_at = k;
      break;
    }
    if (tid == 0 && k + stages < my_tiles) issue(k + stages);
  }

  if (failed_at >= 0) {
    // A stage never completed: report, wait (bounded) for the copies still in flight
    // so none lands after the CTA has left, and return without publishing partials.
    if (tid == 0) {
      set_status(P.status, MB_STATUS_TIMEOUT);
      const long long last = (failed_at - 1 + stages) < (my_tiles - 1) ? (failed_at - 1 + stages) : (my_tiles - 1);
      for (long long j = failed_at; j <= last; ++j)
        mbar_wait_bounded(&bars[j % stages], static_cast<uint32_t>((j / stages) & 1));
    }
    __syncthreads();
    return;
  }

  // ---- remainder rows (fewer than one tile per CTA), plain loads -----------------
  const long long tail0 = P.nfull * TILE;
  for (long long r = tail0 + b * THREADS + tid; r < P.n; r += G * THREADS) {
    RowLoader ld{&P, r};
    process_rows(P, ld, 1u, acc, cnt, s_sum, s_touch, smem, bad_probe, bad_group);
  }

  if (bad_probe) set_status(P.status, MB_STATUS_PROBE_RANGE);
  if (bad_group) set_status(P.status, MB_STATUS_GROUP_RANGE);

  // ---- publish -------------------------------------------------------------------
  const int lane = tid & 31, warp = tid >> 5;
  if (P.gmode == kGroupScalar || P.count != nullptr) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_down_sync(0xffffffffu, acc, o);
      cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    }
    if (lane == 0) {
      s_red[warp] = acc;
      s_red[NWARPS + warp] = cnt;
    }
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long ta = 0, tc = 0;
    for (int w = 0; w < NWARPS; ++w) {
      ta += s_red[w];
      tc += s_red[NWARPS + w];
    }
    if (P.gmode == kGroupScalar && ta != 0) atomicAdd(static_cast<unsigned long long*>(P.res), ta);
    if (P.count != nullptr && tc != 0) {
      if (P.count32)
        atomicAdd(static_cast<int*>(P.count), static_cast<int>(tc));
      else
        atomicAdd(static_cast<unsigned long long*>(P.count), tc);
    }
  }
  if (P.gmode == kGroupSmem) {
    for (int g = tid; g < P.total_val; g += THREADS)
      if ((s_touch[g >> 5] >> (g & 31)) & 1u) atomicAdd(group_sum_ptr(P, g), s_sum[g]);
  }
}

// ---- host launcher ----------------------------------------------------------------

using KernelFn = void (*)(StarPlan);

struct Variant {
  int threads, vpt;
  KernelFn fn;
};

static const Variant kVariants[] = {
    {128, 1, star_kernel<128, 1>}, {128, 2, star_kernel<128, 2>}, {128, 4, star_kernel<128, 4>},
    {256, 1, star_kernel<256, 1>}, {256, 2, star_kernel<256, 2>}, {256, 4, star_kernel<256, 4>},
    {512, 1, star_kernel<512, 1>}, {512, 2, star_kernel<512, 2>}, {512, 4, star_kernel<512, 4>},
};

static const Variant* find_variant(int threads, int vpt) {
  for (const Variant& v : kVariants)
    if (v.threads == threads && v.vpt == vpt) return &v;
  return nullptr;
}

int star_init_device(const DeviceState& ds) {
  for (const Variant& v : kVariants) {
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(v.fn),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         ds.max_smem_optin - 2048);
    if (e != cudaSuccess) return MB_ERR_CUDA;
  }
  return MB_OK;
}

static int add_col(StarPlan& P, const int* c) {
  for (int i = 0; i < P.ncols; ++i)
    if (P.col[i] == c) return i;
  P.col[P.ncols] = c;
  return P.ncols++;
}

static int round_up(int x, int a) { return (x + a - 1) / a * a; }

// Lay out shared memory for `stages` stages; returns total bytes.
static int layout_smem(StarPlan& P, int tile, int stages, bool stage_bitmaps) {
  int off = 128;  // mbarriers (<= 8 x 8 bytes)
  P.smem_groups_off = off;
  if (P.gmode == kGroupSmem) off += round_up(8 * P.total_val + 4 * ((P.total_val + 31) / 32), 128);
  int bm_total = 0;
  for (int p = 0; p < P.np; ++p) {
    P.p_bm_off[p] = -1;
    P.p_bm_words[p] = 0;
    if (!stage_bitmaps) continue;
    const int words = (P.p_slots[p] + 31) / 32;
    const bool can_derive = P.p_layout[p] == MB_HT_KEY;
    const bool have = P.p_presence[p] != nullptr || can_derive;
    if (!have || words * 4 > kBitmapSmemMaxBytes || bm_total + words * 4 > kBitmapSmemTotalBytes) continue;
    P.p_bm_off[p] = off;
    P.p_bm_words[p] = words;
    off += round_up(words * 4, 16);
    bm_total += words * 4;
  }
  off = round_up(off, 128);
  P.smem_stage_off = off;
  P.stage_bytes = P.ncols * tile * 4;
  P.stages = stages;
  P.smem_total = off + stages * P.stage_bytes;
  return P.smem_total;
}

int launch_star(const mb_star_args* a, cudaStream_t stream, int count32) {
  if (a == nullptr) return MB_ERR_ARG;
  if (a->num_rows < 0) return MB_ERR_ARG;
  if (a->num_filters < 0 || a->num_filters > MB_MAX_FILTERS) return MB_ERR_ARG;
  if (a->num_probes < 0 || a->num_probes > MB_MAX_PROBES) return MB_ERR_ARG;
  if (a->aggr[0] == nullptr) return MB_ERR_ARG;
  if (a->agg_op < MB_AGG_SUM || a->agg_op > MB_AGG_MUL_PAYLOAD) return MB_ERR_ARG;
  const bool two_cols = a->agg_op == MB_AGG_SUB || a->agg_op == MB_AGG_MUL;
  if (two_cols && a->aggr[1] == nullptr) return MB_ERR_ARG;
  if (a->agg_op == MB_AGG_MUL_PAYLOAD && (a->num_probes < 1 || a->probe[0].layout == MB_HT_KEY)) return MB_ERR_ARG;
  if (a->res == nullptr || !aligned8(a->res)) return a->res == nullptr ? MB_ERR_ARG : MB_ERR_ALIGN;
  if (a->res_layout < MB_RES_SCALAR || a->res_layout > MB_RES_DENSE) return MB_ERR_ARG;
  if (a->res_layout != MB_RES_SCALAR && a->total_val <= 0) return MB_ERR_ARG;
  if (a->count != nullptr && !count32 && !aligned8(a->count)) return MB_ERR_ALIGN;

  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  if (a->num_rows == 0) return MB_OK;

  StarPlan P;
  memset(&P, 0, sizeof(P));
  P.n = a->num_rows;
  P.nf = a->num_filters;
  for (int f = 0; f < P.nf; ++f) {
    const mb_filter& F = a->filter[f];
    if (F.col == nullptr || F.mode < MB_FILTER_EQ || F.mode > MB_FILTER_EQ_OR_EQ) return MB_ERR_ARG;
    P.f_col[f] = add_col(P, F.col);
    P.f_mode[f] = F.mode;
    P.f_c1[f] = F.c1;
    P.f_c2[f] = F.c2;
  }
  P.np = a->num_probes;
  for (int p = 0; p < P.np; ++p) {
    const mb_probe& Q = a->probe[p];
    if (Q.fkey == nullptr || Q.ht == nullptr || Q.num_slots <= 0) return MB_ERR_ARG;
    if (Q.layout < MB_HT_KEY || Q.layout > MB_HT_VAL_OFF) return MB_ERR_ARG;
    if (Q.layout != MB_HT_KEY && !aligned8(Q.ht)) return MB_ERR_ALIGN;
    const int rs = Q.res_slot;
    if (rs >= 0 && ((a->res_layout == MB_RES_ENGINE6 && rs > 3) || (a->res_layout == MB_RES_CRYSTAL4 && rs > 1)))
      return MB_ERR_ARG;
    P.p_col[p] = add_col(P, Q.fkey);
    P.p_ht[p] = Q.ht;
    P.p_slots[p] = Q.num_slots;
    P.p_kmin[p] = Q.key_min;
    P.p_layout[p] = Q.layout;
    P.p_min[p] = Q.min_val;
    P.p_mul[p] = Q.unique_val;
    P.p_res_slot[p] = (a->res_layout == MB_RES_ENGINE6 || a->res_layout == MB_RES_CRYSTAL4) ? rs : -1;
    P.p_presence[p] = Q.presence;
  }
  P.a_col[0] = add_col(P, a->aggr[0]);
  P.a_col[1] = two_cols ? add_col(P, a->aggr[1]) : 0;
  P.agg_op = a->agg_op;
  P.total_val = a->res_layout == MB_RES_SCALAR ? 1 : a->total_val;
  P.group_bias = a->group_bias;
  P.res_layout = a->res_layout;
  P.res = a->res;
  P.count = a->count;
  P.count32 = count32;
  P.count_after = a->count_after < 0 ? -1 : a->count_after;
  P.status = ds->status;

  if (a->gpu_cache != nullptr) {
    const int ss = a->segment_size;
    if (ss <= 0 || (ss & (ss - 1)) != 0) return MB_ERR_ARG;
    if (!aligned16(a->gpu_cache)) return MB_ERR_ALIGN;
    P.gpu_cache = a->gpu_cache;
    P.seg_group = a->segment_group;
    P.start_offset = a->start_offset;
    P.seg_shift = __builtin_ctz(static_cast<unsigned>(ss));
  }

  // ---- variant and shared-memory plan ------------------------------------------
  int threads = a->threads ? a->threads : (P.res_layout == MB_RES_SCALAR ? 256 : 512);
  int ipt = a->items_per_thread ? a->items_per_thread : (threads == 512 ? 4 : 8);
  if (ipt % 4 != 0) return MB_ERR_ARG;
  const Variant* var = find_variant(threads, ipt / 4);
  if (var == nullptr) return MB_ERR_ARG;
  const int tile = threads * ipt;
  if (P.gpu_cache != nullptr && (1 << P.seg_shift) < tile) return MB_ERR_ARG;

  bool direct_aligned = true;
  for (int c = 0; c < P.ncols; ++c) direct_aligned = direct_aligned && aligned16(P.col[c]);
  const bool use_tiles = P.gpu_cache != nullptr || direct_aligned;
  P.nfull = use_tiles ? P.n / tile : 0;

  P.gmode = P.res_layout == MB_RES_SCALAR ? kGroupScalar
            : (P.total_val <= kSmemGroupMax ? kGroupSmem : kGroupGlobal);
  const int budget = ds->max_smem_optin - 2048 - 2 * 8 * (threads / 32);
  int stages = a->stages ? a->stages : 4;
  if (stages < 2 || stages > kMaxStages) return MB_ERR_ARG;
  int smem = layout_smem(P, tile, stages, true);
  while (smem > budget && P.stages > 2) smem = layout_smem(P, tile, P.stages - 1, true);
  if (smem > budget && P.gmode == kGroupSmem) {
    P.gmode = kGroupGlobal;
    smem = layout_smem(P, tile, stages, true);
    while (smem > budget && P.stages > 2) smem = layout_smem(P, tile, P.stages - 1, true);
  }
  if (smem > budget) smem = layout_smem(P, tile, 2, false);
  if (smem > budget) return MB_ERR_SIZE;

  int grid = a->grid;
  if (grid <= 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, var->fn, threads, smem) != cudaSuccess)
      return MB_ERR_CUDA;
    if (per_sm < 1) per_sm = 1;
    grid = ds->num_sms * per_sm;
  }
  long long want = P.nfull > 0 ? P.nfull : (P.n + threads - 1) / threads;
  if (want < 1) want = 1;
  if (grid > want) grid = static_cast<int>(want);

  var->fn<<<grid, threads, smem, stream>>>(P);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

}  // namespace mb
