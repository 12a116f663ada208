// batch.cu — batched multi-query star execution (see mb_batch_run in mordred_b200.h).
//
// A batch of up to 256 queries is answered by one scan of the fact table:
//   * a producer warp streams fact tiles (the union of the columns the batch reads) into
//     a ring of shared-memory stages with 1-D bulk copies (cp.async.bulk, no multicast);
//   * per row, each needed dimension is looked up once in its packed attribute table (PAT,
//     one 32-bit word per hash slot: bit 31 present, attribute fields below) and the word
//     replaces the key in the stage;
//   * predicates are evaluated for all queries at once: for every attribute some query
//     constrains, a table built per batch maps each value of the queries' range hull to
//     the bitmask of queries accepting it (queries that do not constrain the attribute
//     accept every value), and a table over the 16 dimension-presence patterns does the
//     same for the dimensions each query needs; a row ANDs one mask per attribute and
//     visits only the queries left set;
//   * a visited (row, query) pair adds its 64-bit value to the query's scalar (shared
//     memory), its shared-memory group array (small group counts, flushed once per CTA)
//     or its group array in L2.
// A query's result equals its lone run through mb_star_query with filtered hash tables:
// with unique dimension keys, "the key is in the filtered table" is "the row's
// attributes pass the filter", and the payload is the attribute itself; sums are
// integers, so the order of additions cannot change a bit.
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace mb {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kBatchStages = 8;
constexpr int kMaxPredFields = 8;
constexpr int kMaskWordsMax = MB_BATCH_MAX_QUERIES / 32;
constexpr int kSmemTableMaxEntries = 512;  // predicate tables up to this many values sit in shared memory
constexpr int kMatchListCap = 1024;        // (row, query) pairs a consumer warp collects before aggregating

// Compact per-query descriptor carried in the launch parameters (88 bytes).
struct BQ {
  uint8_t np, nk, agg_op, res_layout;
  uint8_t req, pad[3];
  uint16_t pf[MB_BATCH_MAX_PREDS];
  int plo[MB_BATCH_MAX_PREDS], phi[MB_BATCH_MAX_PREDS];
  uint16_t af[2], kf[2];
  int kmin[2], kmul[2];
  int total_val;
  int smem_off;  // byte offset of this query's shared-memory group array, -1 = L2 atomics
  void* res;
};
static_assert(sizeof(BQ) == 88, "descriptor size");

struct BatchPlan {
  long long n, nfull;
  int ncols;                       // staged fact columns
  const int* col[MB_NUM_FACT_COLS];
  int cidx[13];                    // row-schema column -> stage column (-1: absent)
  int ndims;
  int dim_list[4];
  int key_stage[4];
  const unsigned* pat[4];
  int pat_slots[4], pat_kmin[4];
  int nq, nwords;
  int nfields;                     // attributes some query constrains
  int f_code[kMaxPredFields], f_min[kMaxPredFields], f_n[kMaxPredFields];
  int f_smem_off[kMaxPredFields];  // byte offset of the table in shared memory, -1: workspace
  long long f_goff[kMaxPredFields];// word offset of the table in the workspace
  unsigned outside[kMaxPredFields][kMaskWordsMax];  // mask for values outside the hull
  unsigned pres_mask[16][kMaskWordsMax];
  unsigned* tables;                // workspace
  long long table_entries;
  int stages, stage_words;
  int smem_acc_off, smem_desc_off, smem_pres_off, smem_out_off, smem_tab_off, smem_tab_words, smem_list_off;
  int smem_groups_off, smem_groups_words, smem_stage_off;
  unsigned int* status;
  const int* fact_all[MB_NUM_FACT_COLS];
  BQ q[MB_BATCH_MAX_QUERIES];
};
static_assert(sizeof(BatchPlan) < 32000, "launch parameter limit");

__device__ __forceinline__ int bslot(int key, int slots, int kmin) {
  const int d = static_cast<int>(static_cast<unsigned>(key) - static_cast<unsigned>(kmin));
  if (static_cast<unsigned>(d) < static_cast<unsigned>(slots)) return d;
  if (static_cast<unsigned>(d) < 2u * static_cast<unsigned>(slots)) return d - slots;
  return d % slots;
}

__device__ __forceinline__ int field_value(int v, int code) {
  const int width = code & 63;
  if (width >= 32) return v;
  const int shift = (code >> 6) & 31;
  return static_cast<int>((static_cast<unsigned>(v) >> shift) & ((1u << width) - 1u));
}

__device__ __forceinline__ void bmbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ unsigned long long batch_value(const BQ& Q, int a0, int a1) {
  int v;
  if (Q.agg_op == MB_AGG_SUM)
    v = a0;
  else if (Q.agg_op == MB_AGG_SUB)
    v = static_cast<int>(static_cast<unsigned>(a0) - static_cast<unsigned>(a1));
  else
    v = static_cast<int>(static_cast<unsigned>(a0) * static_cast<unsigned>(a1));
  return static_cast<unsigned long long>(static_cast<long long>(v));
}

__device__ __forceinline__ unsigned long long* batch_sum_ptr(const BQ& Q, int g) {
  if (Q.res_layout == MB_RES_CRYSTAL4) return reinterpret_cast<unsigned long long*>(static_cast<int*>(Q.res) + 4 * g + 2);
  return static_cast<unsigned long long*>(Q.res) + g;
}

// Add one (row, query) match: `get(code)` reads a field of the row.
template <class Get>
__device__ __forceinline__ void batch_match(const BQ& Q, int qi, Get get, unsigned long long* s_acc,
                                            unsigned char* smem, bool& bad_group) {
  const unsigned long long w = batch_value(Q, get(Q.af[0]), Q.agg_op != MB_AGG_SUM ? get(Q.af[1]) : 0);
  if (Q.res_layout == MB_RES_SCALAR) {
    atomicAdd(&s_acc[qi], w);
    return;
  }
  unsigned hh = 0;
  int k0 = 0, k1 = 0;
  if (Q.nk > 0) {
    k0 = get(Q.kf[0]);
    hh += (static_cast<unsigned>(k0) - static_cast<unsigned>(Q.kmin[0])) * static_cast<unsigned>(Q.kmul[0]);
  }
  if (Q.nk > 1) {
    k1 = get(Q.kf[1]);
    hh += (static_cast<unsigned>(k1) - static_cast<unsigned>(Q.kmin[1])) * static_cast<unsigned>(Q.kmul[1]);
  }
  int g = static_cast<int>(hh);
  if (static_cast<unsigned>(g) >= static_cast<unsigned>(Q.total_val)) g = g % Q.total_val;
  if (g < 0) {
    bad_group = true;
    return;
  }
  int* res = static_cast<int*>(Q.res);
  if (Q.smem_off >= 0) {
    // per-CTA partial; the first row of a group in this CTA writes the group's keys
    unsigned long long* s_sum = reinterpret_cast<unsigned long long*>(smem + Q.smem_off);
    uint32_t* s_touch = reinterpret_cast<uint32_t*>(smem + Q.smem_off + 8 * Q.total_val);
    atomicAdd(&s_sum[g], w);
    const uint32_t bit = 1u << (g & 31);
    if (!(s_touch[g >> 5] & bit) && !(atomicOr(&s_touch[g >> 5], bit) & bit) && Q.res_layout == MB_RES_CRYSTAL4) {
      if (Q.nk > 0) res[4 * g] = k0;
      if (Q.nk > 1) res[4 * g + 1] = k1;
    }
    return;
  }
  if (Q.res_layout == MB_RES_CRYSTAL4) {
    if (Q.nk > 0) res[4 * g] = k0;
    if (Q.nk > 1) res[4 * g + 1] = k1;
  }
  atomicAdd(batch_sum_ptr(Q, g), w);
}

// The queries accepting one row: presence mask AND one mask per constrained attribute.
// `get(code)` reads a field of the row.
template <int NWM, class Get>
__device__ __forceinline__ void batch_row_mask(const BatchPlan& P, unsigned pres, Get get, const unsigned* s_pres,
                                               const unsigned* s_out, const unsigned char* smem, unsigned (&m)[NWM]) {
#pragma unroll
  for (int w = 0; w < NWM; ++w) m[w] = s_pres[pres * kMaskWordsMax + w];
  for (int f = 0; f < P.nfields; ++f) {
    unsigned any = 0;
#pragma unroll
    for (int w = 0; w < NWM; ++w) any |= m[w];
    if (!any) return;
    const int v = get(P.f_code[f]) - P.f_min[f];
    const unsigned* t;
    if (static_cast<unsigned>(v) < static_cast<unsigned>(P.f_n[f]))
      t = P.f_smem_off[f] >= 0 ? reinterpret_cast<const unsigned*>(smem + P.f_smem_off[f]) + v * P.nwords
                               : P.tables + P.f_goff[f] + static_cast<long long>(v) * P.nwords;
    else
      t = s_out + f * kMaskWordsMax;
    if (NWM >= 4) {
#pragma unroll
      for (int w = 0; w < NWM; w += 4) {
        const uint4 u = *reinterpret_cast<const uint4*>(t + w);
        m[w] &= u.x;
        m[w + 1] &= u.y;
        m[w + 2] &= u.z;
        m[w + 3] &= u.w;
      }
    } else {
#pragma unroll
      for (int w = 0; w < NWM; ++w) m[w] &= t[w];
    }
  }
}

// Every query a row's mask selects, processed by the lane that owns the row.
template <int NWM, class Get>
__device__ __forceinline__ void batch_row(const BatchPlan& P, unsigned pres, Get get, const BQ* s_desc,
                                          const unsigned* s_pres, const unsigned* s_out, unsigned long long* s_acc,
                                          unsigned char* smem, bool& bad_group) {
  unsigned m[NWM];
  batch_row_mask<NWM>(P, pres, get, s_pres, s_out, smem, m);
#pragma unroll
  for (int w = 0; w < NWM; ++w) {
    unsigned bits = m[w];
    while (bits) {
      const int qi = w * 32 + __ffs(bits) - 1;
      bits &= bits - 1;
      batch_match(s_desc[qi], qi, get, s_acc, smem, bad_group);
    }
  }
}

template <int NCW, int ITEMS, int NWM>
__global__ void __launch_bounds__((NCW + 1) * 32, 1) batch_kernel(const __grid_constant__ BatchPlan P) {
  constexpr int WROWS = 32 * ITEMS;
  constexpr int TILE = NCW * WROWS;
  constexpr int NWARPS = NCW + 1;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kBatchStages;
  unsigned long long* s_acc = reinterpret_cast<unsigned long long*>(smem + P.smem_acc_off);
  BQ* s_desc = reinterpret_cast<BQ*>(smem + P.smem_desc_off);
  unsigned* s_pres = reinterpret_cast<unsigned*>(smem + P.smem_pres_off);
  unsigned* s_out = reinterpret_cast<unsigned*>(smem + P.smem_out_off);
  int* stage_base = reinterpret_cast<int*>(smem + P.smem_stage_off);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = P.stages;

  // ---- set-up: accumulators, descriptors, masks, small tables, barriers ------------
  for (int q = tid; q < P.nq; q += NWARPS * 32) s_acc[q] = 0;
  {
    const unsigned* src = reinterpret_cast<const unsigned*>(P.q);
    unsigned* dst = reinterpret_cast<unsigned*>(s_desc);
    for (int w = tid; w < P.nq * static_cast<int>(sizeof(BQ) / 4); w += NWARPS * 32) dst[w] = src[w];
    for (int w = tid; w < 16 * kMaskWordsMax; w += NWARPS * 32) s_pres[w] = (&P.pres_mask[0][0])[w];
    for (int w = tid; w < kMaxPredFields * kMaskWordsMax; w += NWARPS * 32) s_out[w] = (&P.outside[0][0])[w];
    unsigned* g = reinterpret_cast<unsigned*>(smem + P.smem_groups_off);
    for (int w = tid; w < P.smem_groups_words; w += NWARPS * 32) g[w] = 0;
    for (int f = 0; f < P.nfields; ++f) {
      if (P.f_smem_off[f] < 0) continue;
      unsigned* t = reinterpret_cast<unsigned*>(smem + P.f_smem_off[f]);
      const unsigned* s = P.tables + P.f_goff[f];
      for (int w = tid; w < P.f_n[f] * P.nwords; w += NWARPS * 32) t[w] = s[w];
    }
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    mbar_fence_init();
  }
  __syncthreads();

  const long long G = gridDim.x, b = blockIdx.x;
  const long long my_tiles = P.nfull > b ? (P.nfull - 1 - b) / G + 1 : 0;
  bool failed = false, bad_probe = false, bad_group = false;

  if (warp == 0) {
    if (lane == 0) {
      const uint64_t policy = l2_policy_evict_first();
      long long k = 0;
      int s = 0;
      uint32_t phase = 0;
      for (; k < my_tiles; ++k) {
        if (k >= S && !mbar_wait_bounded(&empty[s], phase ^ 1u)) {
          failed = true;
          break;
        }
        const long long r0 = (b + k * G) * static_cast<long long>(TILE);
        int* dst = stage_base + s * P.stage_words;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>(P.ncols) * TILE * 4u);
        for (int c = 0; c < P.ncols; ++c) bulk_g2s(dst + c * TILE, P.col[c] + r0, TILE * 4, &full[s], policy);
        if (++s == S) {
          s = 0;
          phase ^= 1u;
        }
      }
      for (long long j = (k > S ? k - S : 0); j < k; ++j)
        if (!mbar_wait_bounded(&full[j % S], static_cast<uint32_t>((j / S) & 1))) failed = true;
    }
  } else {
    const int cw = warp - 1;
    int s = 0;
    uint32_t phase = 0;
    for (long long k = 0; k < my_tiles; ++k) {
      const bool ok = mbar_wait_bounded(&full[s], phase);
      if (!__all_sync(kFullMask, ok)) {
        failed = true;
        break;
      }
      int* wst = stage_base + s * P.stage_words + cw * WROWS;
      // ---- dimension words, once per row for the whole batch -------------------
      for (int t = 0; t < P.ndims; ++t) {
        const int d = P.dim_list[t];
        const int* kcol = wst + P.key_stage[d] * TILE;
        int* out = wst + P.cidx[MB_COL_DIM_S + d] * TILE;
        const unsigned* pat = P.pat[d];
        const int slots = P.pat_slots[d], kmin = P.pat_kmin[d];
        unsigned wv[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS / 4; ++j) {
          const int4 kv = lds128(kcol + (j * 32 + lane) * 4);
          const int keys[4] = {kv.x, kv.y, kv.z, kv.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int h = bslot(keys[e], slots, kmin);
            if (h < 0) {
              bad_probe = true;
              wv[4 * j + e] = 0;
            } else {
              wv[4 * j + e] = __ldg(pat + h);
            }
          }
        }
#pragma unroll
        for (int j = 0; j < ITEMS / 4; ++j) {
          int4 o;
          o.x = static_cast<int>(wv[4 * j]);
          o.y = static_cast<int>(wv[4 * j + 1]);
          o.z = static_cast<int>(wv[4 * j + 2]);
          o.w = static_cast<int>(wv[4 * j + 3]);
          *reinterpret_cast<int4*>(out + (j * 32 + lane) * 4) = o;
        }
      }
      __syncwarp();
      // ---- query masks row by row; matches go through the warp's list so that every
      // lane aggregates one (row, query) pair at a time -----------------------------
      unsigned* mlist = reinterpret_cast<unsigned*>(smem + P.smem_list_off) + cw * kMatchListCap;
      int lpos = 0;
      auto flush = [&](int n) {
        for (int base = 0; base < n; base += 32) {
          const int idx = base + lane;
          if (idx < n) {
            const unsigned pr = mlist[idx];
            const int row = static_cast<int>(pr >> 16), qi = static_cast<int>(pr & 0xffffu);
            auto get = [&](int code) { return field_value(wst[P.cidx[code >> 11] * TILE + row], code); };
            batch_match(s_desc[qi], qi, get, s_acc, smem, bad_group);
          }
        }
        __syncwarp();
      };
#pragma unroll 1
      for (int i = 0; i < ITEMS; ++i) {
        const int row = ((i >> 2) * 32 + lane) * 4 + (i & 3);
        unsigned pres = 0;
        for (int t = 0; t < P.ndims; ++t) {
          const int d = P.dim_list[t];
          pres |= (static_cast<unsigned>(wst[P.cidx[MB_COL_DIM_S + d] * TILE + row]) >> 31) << d;
        }
        auto get = [&](int code) { return field_value(wst[P.cidx[code >> 11] * TILE + row], code); };
        unsigned m[NWM];
        batch_row_mask<NWM>(P, pres, get, s_pres, s_out, smem, m);
        int cnt = 0;
#pragma unroll
        for (int w = 0; w < NWM; ++w) cnt += __popc(m[w]);
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(kFullMask, incl, o);
          if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(kFullMask, incl, 31);
        if (total == 0) continue;
        if (lpos + total > kMatchListCap) {
          flush(lpos);
          lpos = 0;
        }
        if (total > kMatchListCap) {
          // more matches than the list holds: this row runs lane by lane
#pragma unroll
          for (int w = 0; w < NWM; ++w) {
            unsigned bits = m[w];
            while (bits) {
              const int qi = w * 32 + __ffs(bits) - 1;
              bits &= bits - 1;
              batch_match(s_desc[qi], qi, get, s_acc, smem, bad_group);
            }
          }
          __syncwarp();
          continue;
        }
        int p = lpos + incl - cnt;
#pragma unroll
        for (int w = 0; w < NWM; ++w) {
          unsigned bits = m[w];
          while (bits) {
            const int qi = w * 32 + __ffs(bits) - 1;
            bits &= bits - 1;
            mlist[p++] = (static_cast<unsigned>(row) << 16) | static_cast<unsigned>(qi);
          }
        }
        lpos += total;
        __syncwarp();
      }
      flush(lpos);
      __syncwarp();
      if (lane == 0) bmbar_arrive(&empty[s]);
      if (++s == S) {
        s = 0;
        phase ^= 1u;
      }
    }
    // ---- remainder rows, one per thread, straight from global memory ------------
    if (!failed) {
      for (long long r = P.nfull * TILE + b * (NCW * 32) + (tid - 32); r < P.n; r += G * (NCW * 32)) {
        int dimw[4] = {0, 0, 0, 0};
        uint32_t pr = 0;
        for (int t = 0; t < P.ndims; ++t) {
          const int d = P.dim_list[t];
          const int key_col = d == 0 ? MB_COL_SUPPKEY : d == 1 ? MB_COL_CUSTKEY : d == 2 ? MB_COL_PARTKEY : MB_COL_ORDERDATE;
          const int h = bslot(__ldg(P.fact_all[key_col] + r), P.pat_slots[d], P.pat_kmin[d]);
          if (h < 0) {
            bad_probe = true;
            continue;
          }
          dimw[d] = static_cast<int>(__ldg(P.pat[d] + h));
          pr |= (static_cast<unsigned>(dimw[d]) >> 31) << d;
        }
        auto get = [&](int code) {
          const int c = code >> 11;
          return field_value(c >= MB_COL_DIM_S ? dimw[c - MB_COL_DIM_S] : __ldg(P.fact_all[c] + r), code);
        };
        batch_row<NWM>(P, pr, get, s_desc, s_pres, s_out, s_acc, smem, bad_group);
      }
    }
  }

  if (failed) set_status(P.status, MB_STATUS_TIMEOUT);
  if (bad_probe) set_status(P.status, MB_STATUS_PROBE_RANGE);
  if (bad_group) set_status(P.status, MB_STATUS_GROUP_RANGE);
  __syncthreads();
  for (int q = tid; q < P.nq; q += NWARPS * 32)
    if (s_desc[q].res_layout == MB_RES_SCALAR && s_acc[q] != 0)
      atomicAdd(static_cast<unsigned long long*>(s_desc[q].res), s_acc[q]);
  for (int q = 0; q < P.nq; ++q) {
    const BQ& Q = s_desc[q];
    if (Q.smem_off < 0) continue;
    const unsigned long long* s_sum = reinterpret_cast<const unsigned long long*>(smem + Q.smem_off);
    const uint32_t* s_touch = reinterpret_cast<const uint32_t*>(smem + Q.smem_off + 8 * Q.total_val);
    for (int g = tid; g < Q.total_val; g += NWARPS * 32)
      if ((s_touch[g >> 5] >> (g & 31)) & 1u) atomicAdd(batch_sum_ptr(Q, g), s_sum[g]);
  }
}

// Per-batch query masks: entry (field f, value v), word w holds bit (q - 32w) for every
// query q that accepts f = f_min + v (every one of its predicates on f holds, or it has none).
__global__ void batch_mask_kernel(const __grid_constant__ BatchPlan P) {
  const long long total = P.table_entries * P.nwords;
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int w = static_cast<int>(e % P.nwords);
    long long v = e / P.nwords;
    int f = 0;
    while (f < P.nfields - 1 && v >= P.f_n[f]) v -= P.f_n[f++];
    const int x = P.f_min[f] + static_cast<int>(v);
    const int code = P.f_code[f];
    unsigned bits = 0;
    for (int j = 0; j < 32; ++j) {
      const int qi = 32 * w + j;
      if (qi >= P.nq) break;
      const BQ& Q = P.q[qi];
      bool ok = true;
      for (int p = 0; p < Q.np; ++p)
        if (Q.pf[p] == code && (x < Q.plo[p] || x > Q.phi[p])) ok = false;
      if (ok) bits |= 1u << j;
    }
    P.tables[P.f_goff[f] + v * P.nwords + w] = bits;
  }
}

// ---- PAT build -----------------------------------------------------------------------
__global__ void pat_build_kernel(const int* key, int n, int kmin, int slots, const int* a0, int f0, const int* a1, int f1,
                                 const int* a2, int f2, unsigned* words, unsigned* status) {
  bool bad_slot = false, bad_attr = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int h = bslot(key[i], slots, kmin);
    if (h < 0) {
      bad_slot = true;
      continue;
    }
    unsigned w = 0x80000000u;
    const int* attrs[3] = {a0, a1, a2};
    const int fields[3] = {f0, f1, f2};
    for (int k = 0; k < 3; ++k) {
      if (attrs[k] == nullptr) continue;
      const int width = fields[k] & 63, shift = (fields[k] >> 6) & 31;
      const unsigned v = static_cast<unsigned>(attrs[k][i]);
      if (width < 32 && (v >> width) != 0) {
        bad_attr = true;
        continue;
      }
      w |= v << shift;
    }
    words[h] = w;
  }
  if (bad_slot) set_status(status, MB_STATUS_PROBE_RANGE);
  if (bad_attr) set_status(status, MB_STATUS_GROUP_RANGE);
}

// ---- host ----------------------------------------------------------------------------
using BatchFn = void (*)(BatchPlan);
struct BatchVariant {
  int warps, items, nwm;
  BatchFn fn;
};
#define MB_BATCH_VARIANTS(W, I) \
  {W, I, 1, batch_kernel<W, I, 1>}, {W, I, 2, batch_kernel<W, I, 2>}, {W, I, 4, batch_kernel<W, I, 4>}, \
      {W, I, 8, batch_kernel<W, I, 8>}
static const BatchVariant kBatchVariants[] = {
    MB_BATCH_VARIANTS(4, 4), MB_BATCH_VARIANTS(8, 4), MB_BATCH_VARIANTS(16, 4), MB_BATCH_VARIANTS(8, 8),
};

static bool field_ok(int code) {
  const int col = code >> 11, width = code & 63, shift = (code >> 6) & 31;
  return col >= 0 && col <= MB_COL_DIM_D && width >= 1 && width <= 32 && (width == 32 || shift + width <= 32) &&
         code < 65536;
}

int batch_init_device(const DeviceState& ds) {
  for (const BatchVariant& v : kBatchVariants)
    if (cudaFuncSetAttribute(reinterpret_cast<const void*>(v.fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                             ds.max_smem_optin - 2048) != cudaSuccess)
      return MB_ERR_CUDA;
  return MB_OK;
}

// Fill everything but the shared-memory layout; returns MB_OK or an error.
static int plan_batch(const mb_batch_args* a, BatchPlan& P) {
  if (a == nullptr || a->num_queries < 1 || a->num_queries > MB_BATCH_MAX_QUERIES || a->queries == nullptr)
    return MB_ERR_ARG;
  if (a->num_rows < 0) return MB_ERR_ARG;
  memset(&P, 0, sizeof(P));
  P.n = a->num_rows;
  P.nq = a->num_queries;
  // mask words per entry, rounded to 1, 2, 4 or 8 so table entries stay 16-byte aligned
  const int words = (P.nq + 31) / 32;
  P.nwords = words <= 1 ? 1 : words <= 2 ? 2 : words <= 4 ? 4 : 8;
  bool fact_used[MB_NUM_FACT_COLS] = {false};
  unsigned dims_used = 0;
  auto note_field = [&](int code) -> bool {
    if (!field_ok(code)) return false;
    const int col = code >> 11;
    if (col < MB_NUM_FACT_COLS) {
      if (a->fact[col] == nullptr) return false;
      fact_used[col] = true;
    } else {
      dims_used |= 1u << (col - MB_COL_DIM_S);
    }
    return true;
  };
  for (int qi = 0; qi < P.nq; ++qi) {
    const mb_batch_query& q = a->queries[qi];
    BQ& d = P.q[qi];
    if (q.num_preds < 0 || q.num_preds > MB_BATCH_MAX_PREDS || q.num_keys < 0 || q.num_keys > 2) return MB_ERR_ARG;
    if (q.agg_op < MB_AGG_SUM || q.agg_op > MB_AGG_MUL || q.res == nullptr) return MB_ERR_ARG;
    if (q.res_layout != MB_RES_SCALAR && q.res_layout != MB_RES_CRYSTAL4 && q.res_layout != MB_RES_DENSE)
      return MB_ERR_ARG;
    if (q.res_layout != MB_RES_SCALAR && q.total_val <= 0) return MB_ERR_ARG;
    if (!aligned8(q.res)) return MB_ERR_ALIGN;
    if (q.dims_required < 0 || q.dims_required > 15) return MB_ERR_ARG;
    d.np = static_cast<uint8_t>(q.num_preds);
    d.nk = static_cast<uint8_t>(q.res_layout == MB_RES_SCALAR ? 0 : q.num_keys);
    d.agg_op = static_cast<uint8_t>(q.agg_op);
    d.res_layout = static_cast<uint8_t>(q.res_layout);
    d.req = static_cast<uint8_t>(q.dims_required);
    d.smem_off = -1;
    dims_used |= static_cast<unsigned>(q.dims_required);
    for (int p = 0; p < q.num_preds; ++p) {
      if (!note_field(q.pred_field[p])) return MB_ERR_ARG;
      d.pf[p] = static_cast<uint16_t>(q.pred_field[p]);
      d.plo[p] = q.pred_lo[p];
      d.phi[p] = q.pred_hi[p];
    }
    for (int k = 0; k < (q.agg_op == MB_AGG_SUM ? 1 : 2); ++k) {
      if (!note_field(q.agg_field[k])) return MB_ERR_ARG;
      d.af[k] = static_cast<uint16_t>(q.agg_field[k]);
    }
    for (int k = 0; k < d.nk; ++k) {
      if (!note_field(q.key_field[k])) return MB_ERR_ARG;
      d.kf[k] = static_cast<uint16_t>(q.key_field[k]);
      d.kmin[k] = q.key_min[k];
      d.kmul[k] = q.key_mul[k];
    }
    d.total_val = q.res_layout == MB_RES_SCALAR ? 1 : q.total_val;
    d.res = q.res;
  }
  // constrained attributes and the hull of the ranges on each
  int hmin[kMaxPredFields], hmax[kMaxPredFields];
  bool has[kMaxPredFields] = {false};
  for (int qi = 0; qi < P.nq; ++qi) {
    const BQ& d = P.q[qi];
    for (int p = 0; p < d.np; ++p) {
      int f = 0;
      while (f < P.nfields && P.f_code[f] != d.pf[p]) ++f;
      if (f == P.nfields) {
        if (P.nfields == kMaxPredFields) return MB_ERR_SIZE;
        P.f_code[P.nfields++] = d.pf[p];
      }
      if (d.plo[p] > d.phi[p]) continue;  // an empty range accepts nothing, inside or outside the hull
      if (!has[f]) {
        hmin[f] = d.plo[p];
        hmax[f] = d.phi[p];
        has[f] = true;
      } else {
        hmin[f] = d.plo[p] < hmin[f] ? d.plo[p] : hmin[f];
        hmax[f] = d.phi[p] > hmax[f] ? d.phi[p] : hmax[f];
      }
    }
  }
  long long entries = 0;
  for (int f = 0; f < P.nfields; ++f) {
    const long long n = has[f] ? static_cast<long long>(hmax[f]) - hmin[f] + 1 : 1;
    if (n > 65536) return MB_ERR_SIZE;  // attribute ranges wider than 65,536 values
    P.f_min[f] = has[f] ? hmin[f] : 0;
    P.f_n[f] = static_cast<int>(n);
    P.f_goff[f] = entries * P.nwords;
    entries += P.f_n[f];
  }
  P.table_entries = entries;
  // values outside a hull fail every query constraining that attribute
  for (int f = 0; f < P.nfields; ++f)
    for (int qi = 0; qi < P.nq; ++qi) {
      bool constrains = false;
      for (int p = 0; p < P.q[qi].np; ++p) constrains = constrains || P.q[qi].pf[p] == P.f_code[f];
      if (!constrains) P.outside[f][qi / 32] |= 1u << (qi % 32);
    }
  for (int pm = 0; pm < 16; ++pm)
    for (int qi = 0; qi < P.nq; ++qi)
      if ((pm & P.q[qi].req) == P.q[qi].req) P.pres_mask[pm][qi / 32] |= 1u << (qi % 32);

  // dimensions: their keys are staged, their words overwrite the key columns (the date
  // word gets its own column because orderdate is also a field)
  static const int kKeyCol[4] = {MB_COL_SUPPKEY, MB_COL_CUSTKEY, MB_COL_PARTKEY, MB_COL_ORDERDATE};
  for (int d = 0; d < 4; ++d) {
    if (!(dims_used & (1u << d))) continue;
    if (a->dim[d].words == nullptr || a->dim[d].slots <= 0 || a->fact[kKeyCol[d]] == nullptr) return MB_ERR_ARG;
    fact_used[kKeyCol[d]] = true;
  }
  for (int c = 0; c < 13; ++c) P.cidx[c] = -1;
  for (int c = 0; c < MB_NUM_FACT_COLS; ++c) {
    P.fact_all[c] = a->fact[c];
    if (!fact_used[c]) continue;
    if (!aligned16(a->fact[c])) return MB_ERR_ALIGN;
    P.cidx[c] = P.ncols;
    P.col[P.ncols++] = a->fact[c];
  }
  for (int d = 0; d < 4; ++d) {
    if (!(dims_used & (1u << d))) continue;
    P.dim_list[P.ndims++] = d;
    P.key_stage[d] = P.cidx[kKeyCol[d]];
    P.pat[d] = a->dim[d].words;
    P.pat_slots[d] = a->dim[d].slots;
    P.pat_kmin[d] = a->dim[d].key_min;
    P.cidx[MB_COL_DIM_S + d] = d == 3 ? P.ncols : P.key_stage[d];
  }
  // a dimension word that replaces its key makes that key unavailable as a field
  for (int qi = 0; qi < P.nq; ++qi) {
    const BQ& d = P.q[qi];
    auto uses_key = [&](int code) {
      const int col = code >> 11;
      for (int t = 0; t < 3; ++t)
        if ((dims_used & (1u << t)) && col == kKeyCol[t]) return true;
      return false;
    };
    for (int p = 0; p < d.np; ++p)
      if (uses_key(d.pf[p])) return MB_ERR_ARG;
    for (int k = 0; k < (d.agg_op == MB_AGG_SUM ? 1 : 2); ++k)
      if (uses_key(d.af[k])) return MB_ERR_ARG;
    for (int k = 0; k < d.nk; ++k)
      if (uses_key(d.kf[k])) return MB_ERR_ARG;
  }
  return MB_OK;
}

static size_t workspace_bytes(const BatchPlan& P) { return static_cast<size_t>(P.table_entries) * P.nwords * 4; }

}  // namespace mb

using namespace mb;

extern "C" int mb_pat_build(const int* dim_key, int num_rows, int key_min, int slots, const int* attr0, int field0,
                            const int* attr1, int field1, const int* attr2, int field2, unsigned int* words,
                            mb_stream_t stream) {
  if (num_rows == 0) return MB_OK;
  if (dim_key == nullptr || words == nullptr || num_rows < 0 || slots <= 0) return MB_ERR_ARG;
  if ((attr0 && !field_ok(field0)) || (attr1 && !field_ok(field1)) || (attr2 && !field_ok(field2))) return MB_ERR_ARG;
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  int blocks = (num_rows + 255) / 256;
  if (blocks > ds->num_sms * 8) blocks = ds->num_sms * 8;
  pat_build_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(dim_key, num_rows, key_min, slots, attr0,
                                                                          field0, attr1, field1, attr2, field2, words,
                                                                          ds->status);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

extern "C" size_t mb_batch_workspace_bytes(const mb_batch_args* a) {
  static BatchPlan P;  // large; host-side scratch for sizing only
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (plan_batch(a, P) != MB_OK) return 0;
  return workspace_bytes(P);
}

extern "C" int mb_batch_run(const mb_batch_args* a, mb_stream_t stream) {
  BatchPlan* Pp = new BatchPlan;  // ~25 KB of launch parameters, kept off the host stack
  struct Free {
    BatchPlan* p;
    ~Free() { delete p; }
  } guard{Pp};
  BatchPlan& P = *Pp;
  int e = plan_batch(a, P);
  if (e != MB_OK) return e;
  if (P.n == 0) return MB_OK;
  if (workspace_bytes(P) > 0 &&
      (a->workspace == nullptr || a->workspace_bytes < workspace_bytes(P) || !aligned16(a->workspace)))
    return a->workspace == nullptr || a->workspace_bytes < workspace_bytes(P) ? MB_ERR_SIZE : MB_ERR_ALIGN;
  P.tables = static_cast<unsigned*>(a->workspace);
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  P.status = ds->status;

  const int threads = a->threads ? a->threads : 256;
  const int items = a->items_per_thread ? a->items_per_thread : 4;
  const int nwm = P.nwords;
  const BatchVariant* var = nullptr;
  for (const BatchVariant& v : kBatchVariants)
    if (v.warps * 32 == threads && v.items == items && v.nwm == nwm) var = &v;
  if (var == nullptr) return MB_ERR_ARG;
  const int tile = threads * items;
  P.nfull = P.n / tile;
  P.stage_words = (P.ncols + ((P.ndims && P.dim_list[P.ndims - 1] == 3) ? 1 : 0)) * tile;
  int stages = a->stages ? a->stages : 2;
  if (stages < 2 || stages > kBatchStages) return MB_ERR_ARG;

  // shared memory: barriers | scalars | descriptors | presence masks | outside masks |
  // small predicate tables | small group arrays | stage ring
  int off = 2 * kBatchStages * 8;
  P.smem_acc_off = off;
  off += 8 * P.nq;
  off = (off + 15) / 16 * 16;
  P.smem_desc_off = off;
  off += static_cast<int>(sizeof(BQ)) * P.nq;
  off = (off + 15) / 16 * 16;
  P.smem_pres_off = off;
  off += 16 * kMaskWordsMax * 4;
  P.smem_out_off = off;
  off += kMaxPredFields * kMaskWordsMax * 4;
  P.smem_tab_off = off;
  for (int f = 0; f < P.nfields; ++f) {
    P.f_smem_off[f] = -1;
    if (P.f_n[f] <= kSmemTableMaxEntries) {
      P.f_smem_off[f] = off;
      off += (P.f_n[f] * P.nwords * 4 + 15) / 16 * 16;
    }
  }
  P.smem_list_off = off;
  off += (threads / 32) * kMatchListCap * 4;
  const int budget = ds->max_smem_optin - 2048;
  auto total_smem = [&](int base, int st) { return (base + 127) / 128 * 128 + st * P.stage_words * 4; };
  while (total_smem(off, stages) > budget && stages > 2) --stages;
  if (total_smem(off, stages) > budget) return MB_ERR_SIZE;
  P.stages = stages;
  // small group arrays (<= 1,024 groups) to shared memory, smallest first, within the budget
  P.smem_groups_off = off;
  int groups_bytes = 0;
  const int group_cap = a->smem_group_bytes < 0 ? 65536 : a->smem_group_bytes;
  for (int pass_total = 1; pass_total <= 1024; pass_total *= 2) {
    for (int qi = 0; qi < P.nq; ++qi) {
      BQ& d = P.q[qi];
      if (d.res_layout == MB_RES_SCALAR || d.smem_off >= 0 || d.total_val > pass_total) continue;
      const int bytes = (8 * d.total_val + 4 * ((d.total_val + 31) / 32) + 15) / 16 * 16;
      if (groups_bytes + bytes > group_cap || total_smem(off + groups_bytes + bytes, stages) > budget) continue;
      d.smem_off = off + groups_bytes;
      groups_bytes += bytes;
    }
  }
  P.smem_groups_words = groups_bytes / 4;
  P.smem_stage_off = (off + groups_bytes + 127) / 128 * 128;
  const int smem = total_smem(off + groups_bytes, stages);

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (P.table_entries > 0) {
    const long long work = P.table_entries * P.nwords;
    long long blocks = (work + 255) / 256;
    if (blocks > ds->num_sms * 8) blocks = ds->num_sms * 8;
    batch_mask_kernel<<<static_cast<int>(blocks), 256, 0, st>>>(P);
    if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
    note_launches(1);
  }
  int grid = a->grid;
  if (grid <= 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, var->fn, threads + 32, smem) != cudaSuccess)
      return MB_ERR_CUDA;
    grid = ds->num_sms * (per_sm < 1 ? 1 : per_sm);
  }
  long long want = P.nfull > 0 ? P.nfull : (P.n + threads - 1) / threads;
  if (want < 1) want = 1;
  if (grid > want) grid = static_cast<int>(want);
  var->fn<<<grid, threads + 32, smem, st>>>(P);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}
