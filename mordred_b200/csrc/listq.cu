// listq.cu — the fused star pipeline over an offset list: the rows a previous operator
// selected (on the GPU by mb_star_select, or on the CPU) arrive as a list of physical fact
// rows, possibly with the dimension rows earlier joins matched them with, and are
// filtered, probed, grouped and aggregated here.
//
// Restates the offset-list ("GPU3") forms of the engine's fused kernels:
//   filter_probe_group_by_GPU3  src/gpudb/GPUProcessing.h:157-273
//   probe_group_by_GPU3         GPUProcessing.h:393-494
//   groupByGPU                  GPUProcessing.h:1385-1470
//   aggregationGPU              GPUProcessing.h:1472-1524
//   probe_aggr_GPU3             GPUProcessing.h:1610-1673
//   filter_probe_aggr_GPU3      GPUProcessing.h:1778-1846
// Row k of the call reads every fact column at the physical row rows[k] (through the
// segment cache: gpuCache[col_idx[row >> 20] << 20 | row & (2^20 - 1)], BlockLibrary.cuh:
// 543-592); a probe either looks the row's key up in a hash table, or — layout MB_HT_PASS —
// takes the group value an earlier join found: the dimension column `ht` read at the
// dimension row fkey[k] (BlockReadFilteredOffset, BlockLibrary.cuh:484-541).
//
// The rows of a list are gathers, not a stream, so this kernel is a plain grid-stride loop
// (each thread keeps kListItems rows in flight) with the star kernel's group accumulation:
// 64-bit sums in a shared-memory group array flushed once per CTA, or L2 atomics for large
// group arrays; scalars reduced per CTA.
#include <cstring>

#include "star.cuh"

namespace mb {

constexpr int kListItems = 4;
constexpr int kListThreads = 256;

struct ListPlan {
  long long n;
  const int* rows;  // physical fact rows, or null: row k is virtual row k
  int nf;
  const int* f_col[MB_MAX_FILTERS];
  int f_mode[MB_MAX_FILTERS], f_c1[MB_MAX_FILTERS], f_c2[MB_MAX_FILTERS];
  int np;
  const int* p_key[MB_MAX_PROBES];
  const int* p_ht[MB_MAX_PROBES];
  int p_slots[MB_MAX_PROBES], p_kmin[MB_MAX_PROBES], p_layout[MB_MAX_PROBES];
  int p_min[MB_MAX_PROBES], p_mul[MB_MAX_PROBES], p_res_slot[MB_MAX_PROBES];
  const int* a_col[2];
  int agg_op;
  int total_val, group_bias, res_layout;
  void* res;
  unsigned long long* count;
  int count_after;
  int gmode;
  const int* gpu_cache;
  const short* seg_group;
  long long start_offset;
  int seg_shift;
  unsigned int* status;
};

__device__ __forceinline__ bool list_pass(int x, int mode, int c1, int c2) {
  if (mode == MB_FILTER_BETWEEN) return x >= c1 && x <= c2;
  if (mode == MB_FILTER_EQ) return x == c1;
  return x == c1 || x == c2;
}

// Where row k of the call lives: (segment, in-segment row) under segment addressing,
// (-1, column index) otherwise.
__device__ __forceinline__ void list_locate(const ListPlan& P, long long k, int& seg, long long& idx) {
  const long long phys = P.rows ? static_cast<long long>(__ldg(P.rows + k)) : k;
  if (P.gpu_cache == nullptr) {
    seg = -1;
    idx = phys;
    return;
  }
  const long long mask = (1ll << P.seg_shift) - 1;
  if (P.rows) {
    seg = static_cast<int>(phys >> P.seg_shift);  // physical rows index the slot arrays directly
  } else {
    const long long vseg = k >> P.seg_shift;
    seg = P.seg_group ? static_cast<int>(P.seg_group[vseg]) : static_cast<int>((P.start_offset + k) >> P.seg_shift);
  }
  idx = phys & mask;
}

__device__ __forceinline__ int list_read(const ListPlan& P, const int* col, int seg, long long idx) {
  if (P.gpu_cache == nullptr) return __ldg(col + idx);
  return __ldg(P.gpu_cache + (static_cast<long long>(__ldg(col + seg)) << P.seg_shift) + idx);
}

// A dimension column at dimension row d (direct, or through the segment cache).
__device__ __forceinline__ int list_read_dim(const ListPlan& P, const int* col, int d) {
  if (P.gpu_cache == nullptr) return __ldg(col + d);
  const int seg = d >> P.seg_shift;
  return __ldg(P.gpu_cache + (static_cast<long long>(__ldg(col + seg)) << P.seg_shift) +
               (d & ((1 << P.seg_shift) - 1)));
}

__device__ __forceinline__ unsigned long long* list_sum_ptr(const ListPlan& P, int h) {
  if (P.res_layout == MB_RES_ENGINE6)
    return reinterpret_cast<unsigned long long*>(static_cast<int*>(P.res) + 6 * h + 4);
  if (P.res_layout == MB_RES_CRYSTAL4)
    return reinterpret_cast<unsigned long long*>(static_cast<int*>(P.res) + 4 * h + 2);
  return static_cast<unsigned long long*>(P.res) + h;
}

__device__ __forceinline__ void list_keys(const ListPlan& P, int h, const int (&gv)[MB_MAX_PROBES]) {
  int* res = static_cast<int*>(P.res);
  const int stride = P.res_layout == MB_RES_ENGINE6 ? 6 : 4;
  for (int p = 0; p < P.np; ++p)
    if (P.p_res_slot[p] >= 0) res[stride * h + P.p_res_slot[p]] = gv[p];
}

__global__ void __launch_bounds__(kListThreads) list_kernel(const __grid_constant__ ListPlan P) {
  extern __shared__ __align__(16) unsigned char lsmem[];
  __shared__ unsigned long long s_red[2 * kListThreads / 32];
  unsigned long long* s_sum = reinterpret_cast<unsigned long long*>(lsmem);
  uint32_t* s_touch = reinterpret_cast<uint32_t*>(lsmem + 8 * P.total_val);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (P.gmode == kGroupSmem) {
    for (int g = tid; g < P.total_val; g += kListThreads) s_sum[g] = 0;
    for (int w = tid; w < (P.total_val + 31) / 32; w += kListThreads) s_touch[w] = 0;
  }
  __syncthreads();
  unsigned long long acc = 0, cnt = 0;
  bool bad_probe = false, bad_group = false;
  const long long stride = static_cast<long long>(gridDim.x) * kListThreads;
  for (long long base = blockIdx.x * static_cast<long long>(kListThreads) * kListItems + tid; base < P.n;
       base += stride * kListItems) {
    // kListItems rows a thread, k = base + i * kListThreads: their gathers are independent
    int seg[kListItems];
    long long idx[kListItems];
    bool ok[kListItems];
#pragma unroll
    for (int i = 0; i < kListItems; ++i) {
      const long long k = base + static_cast<long long>(i) * kListThreads;
      ok[i] = k < P.n;
      seg[i] = 0;
      idx[i] = 0;
      if (ok[i]) list_locate(P, k, seg[i], idx[i]);
    }
    for (int f = 0; f < P.nf; ++f) {
#pragma unroll
      for (int i = 0; i < kListItems; ++i) {
        if (P.count_after == f && ok[i]) ++cnt;
        if (ok[i]) ok[i] = list_pass(list_read(P, P.f_col[f], seg[i], idx[i]), P.f_mode[f], P.f_c1[f], P.f_c2[f]);
      }
    }
    if (P.count_after >= P.nf) {
#pragma unroll
      for (int i = 0; i < kListItems; ++i) cnt += ok[i];
    }
    int gv[kListItems][MB_MAX_PROBES];
    for (int p = 0; p < P.np; ++p) {
#pragma unroll
      for (int i = 0; i < kListItems; ++i) {
        gv[i][p] = 0;
        if (!ok[i]) continue;
        if (P.p_layout[p] == MB_HT_PASS) {
          const long long k = base + static_cast<long long>(i) * kListThreads;
          const int d = __ldg(P.p_key[p] + k);
          if (d < 0 || d >= P.p_slots[p]) {
            bad_probe = true;
            ok[i] = false;
          } else {
            gv[i][p] = list_read_dim(P, P.p_ht[p], d);
          }
          continue;
        }
        const int key = list_read(P, P.p_key[p], seg[i], idx[i]);
        const int dd = static_cast<int>(static_cast<unsigned>(key) - static_cast<unsigned>(P.p_kmin[p]));
        const int h = (static_cast<unsigned>(dd) < static_cast<unsigned>(P.p_slots[p])) ? dd : dd % P.p_slots[p];
        if (h < 0) {
          bad_probe = true;
          ok[i] = false;
        } else if (P.p_layout[p] == MB_HT_KEY) {
          ok[i] = __ldg(P.p_ht[p] + h) != 0;
        } else {
          const unsigned long long s = ldg_u64(P.p_ht[p] + 2ll * h);
          ok[i] = s != 0;
          gv[i][p] = P.p_layout[p] == MB_HT_KEY_VAL ? static_cast<int>(s >> 32) : static_cast<int>(static_cast<unsigned>(s));
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kListItems; ++i) {
      if (!ok[i]) continue;
      if (P.count_after < 0) ++cnt;
      const int a0 = list_read(P, P.a_col[0], seg[i], idx[i]);
      int val;
      if (P.agg_op == MB_AGG_SUM) {
        val = a0;
      } else if (P.agg_op == MB_AGG_MUL_PAYLOAD) {
        val = static_cast<int>(static_cast<unsigned>(a0) * static_cast<unsigned>(gv[i][0]));
      } else {
        const int a1 = list_read(P, P.a_col[1], seg[i], idx[i]);
        val = P.agg_op == MB_AGG_SUB ? static_cast<int>(static_cast<unsigned>(a0) - static_cast<unsigned>(a1))
                                     : static_cast<int>(static_cast<unsigned>(a0) * static_cast<unsigned>(a1));
      }
      const unsigned long long w = static_cast<unsigned long long>(static_cast<long long>(val));
      if (P.gmode == kGroupScalar) {
        acc += w;
        continue;
      }
      unsigned hh = static_cast<unsigned>(P.group_bias);
      for (int p = 0; p < P.np; ++p)
        hh += (static_cast<unsigned>(gv[i][p]) - static_cast<unsigned>(P.p_min[p])) * static_cast<unsigned>(P.p_mul[p]);
      const int h = static_cast<int>(hh) % P.total_val;
      if (h < 0) {
        bad_group = true;
        continue;
      }
      if (P.gmode == kGroupSmem) {
        atomicAdd(&s_sum[h], w);
        const uint32_t bit = 1u << (h & 31);
        if (!(s_touch[h >> 5] & bit) && !(atomicOr(&s_touch[h >> 5], bit) & bit) && P.res_layout != MB_RES_DENSE)
          list_keys(P, h, gv[i]);
      } else {
        if (P.res_layout != MB_RES_DENSE) list_keys(P, h, gv[i]);
        atomicAdd(list_sum_ptr(P, h), w);
      }
    }
  }
  if (bad_probe) set_status(P.status, MB_STATUS_PROBE_RANGE);
  if (bad_group) set_status(P.status, MB_STATUS_GROUP_RANGE);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_down_sync(0xffffffffu, acc, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  if (lane == 0) {
    s_red[warp] = acc;
    s_red[kListThreads / 32 + warp] = cnt;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long ta = 0, tc = 0;
    for (int w = 0; w < kListThreads / 32; ++w) {
      ta += s_red[w];
      tc += s_red[kListThreads / 32 + w];
    }
    if (P.gmode == kGroupScalar && ta != 0) atomicAdd(static_cast<unsigned long long*>(P.res), ta);
    if (P.count != nullptr && tc != 0) atomicAdd(P.count, tc);
  }
  if (P.gmode == kGroupSmem) {
    for (int g = tid; g < P.total_val; g += kListThreads)
      if ((s_touch[g >> 5] >> (g & 31)) & 1u) atomicAdd(list_sum_ptr(P, g), s_sum[g]);
  }
}

int list_init_device(const DeviceState& ds) {
  return cuda_status(cudaFuncSetAttribute(reinterpret_cast<const void*>(list_kernel),
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, ds.max_smem_optin - 2048));
}

int launch_list(const mb_star_args* a, cudaStream_t stream, const DeviceState* ds) {
  ListPlan P;
  memset(&P, 0, sizeof(P));
  P.n = a->num_rows;
  P.rows = a->rows;
  P.nf = a->num_filters;
  for (int f = 0; f < P.nf; ++f) {
    const mb_filter& F = a->filter[f];
    if (F.col == nullptr || F.mode < MB_FILTER_EQ || F.mode > MB_FILTER_EQ_OR_EQ) return MB_ERR_ARG;
    P.f_col[f] = F.col;
    P.f_mode[f] = F.mode;
    P.f_c1[f] = F.c1;
    P.f_c2[f] = F.c2;
  }
  P.np = a->num_probes;
  for (int p = 0; p < P.np; ++p) {
    const mb_probe& Q = a->probe[p];
    if (Q.fkey == nullptr || Q.ht == nullptr || Q.num_slots <= 0) return MB_ERR_ARG;
    if (Q.layout < MB_HT_KEY || Q.layout > MB_HT_PASS) return MB_ERR_ARG;
    if ((Q.layout == MB_HT_KEY_VAL || Q.layout == MB_HT_VAL_OFF) && !aligned8(Q.ht)) return MB_ERR_ALIGN;
    const int rs = Q.res_slot;
    if (rs >= 0 && ((a->res_layout == MB_RES_ENGINE6 && rs > 3) || (a->res_layout == MB_RES_CRYSTAL4 && rs > 1)))
      return MB_ERR_ARG;
    P.p_key[p] = Q.fkey;
    P.p_ht[p] = Q.ht;
    P.p_slots[p] = Q.num_slots;
    P.p_kmin[p] = Q.key_min;
    P.p_layout[p] = Q.layout;
    P.p_min[p] = Q.min_val;
    P.p_mul[p] = Q.unique_val;
    P.p_res_slot[p] = (a->res_layout == MB_RES_ENGINE6 || a->res_layout == MB_RES_CRYSTAL4) ? rs : -1;
  }
  if (a->agg_op == MB_AGG_MUL_PAYLOAD && (P.np < 1 || P.p_layout[0] == MB_HT_KEY)) return MB_ERR_ARG;
  P.a_col[0] = a->aggr[0];
  P.a_col[1] = a->aggr[1];
  P.agg_op = a->agg_op;
  P.total_val = a->res_layout == MB_RES_SCALAR ? 1 : a->total_val;
  P.group_bias = a->group_bias;
  P.res_layout = a->res_layout;
  P.res = a->res;
  P.count = a->count;
  P.count_after = a->count_after < 0 ? -1 : a->count_after;
  P.status = ds->status;
  if (a->gpu_cache != nullptr) {
    const int ss = a->segment_size;
    if (ss <= 0 || (ss & (ss - 1)) != 0) return MB_ERR_ARG;
    P.gpu_cache = a->gpu_cache;
    P.seg_group = a->rows ? nullptr : a->segment_group;
    P.start_offset = a->start_offset;
    P.seg_shift = __builtin_ctz(static_cast<unsigned>(ss));
  }
  int smem = 0;
  if (P.res_layout == MB_RES_SCALAR) {
    P.gmode = kGroupScalar;
  } else if (a->group_mode != 2 && P.total_val <= kSmemGroupMax) {
    P.gmode = kGroupSmem;
    smem = 8 * P.total_val + 4 * ((P.total_val + 31) / 32);
  } else {
    if (a->group_mode == 1) return MB_ERR_SIZE;
    P.gmode = kGroupGlobal;
  }
  const long long per_block = static_cast<long long>(kListThreads) * kListItems;
  long long blocks = (P.n + per_block - 1) / per_block;
  const long long cap = static_cast<long long>(ds->num_sms) * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  list_kernel<<<static_cast<int>(blocks), kListThreads, smem, stream>>>(P);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

}  // namespace mb
