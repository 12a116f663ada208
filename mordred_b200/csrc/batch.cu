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
//   * the (row, query) pairs a warp finds go to a list in shared memory; a full list is
//     aggregated 32 pairs at a time, one per lane, by branch-light code driven by a
//     32-byte per-query descriptor: the pair's 64-bit value is added to the query's
//     scalar or shared-memory group array (flushed once per CTA) or its group array in L2.
// A query's result equals its lone run through mb_star_query with filtered hash tables:
// with unique dimension keys, "the key is in the filtered table" is "the row's
// attributes pass the filter", and the payload is the attribute itself; sums are
// integers, so the order of additions cannot change a bit.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace mb {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kBatchStages = 8;
constexpr int kMaxPredFields = 8;
constexpr int kMaskWordsMax = MB_BATCH_MAX_QUERIES / 32;
constexpr int kSmemTableMaxEntries = 512;  // predicate tables up to this many values sit in shared memory
constexpr int kMatchListMax = 1024;        // (row, query) pairs a consumer warp collects before aggregating
constexpr int kColPad = 4;                 // words between staged columns: the same row of two columns
                                           // falls in different banks (and stays 16-byte aligned)
constexpr int kMaxStageCols = MB_NUM_FACT_COLS + 1;
constexpr int kMaxBreakpoints = 768;       // range end points of wide attributes, over all of them
constexpr int kMaxBuckets = 2048;          // bucket index entries per wide attribute
constexpr int kScalarCopies = 4;           // shared-memory copies of each scalar sum, one per lane mod 4:
                                           // rows of one date (a date-sorted table) match the same
                                           // scalar queries, and same-word atomics of one warp serialise

// Field codes inside the kernel address staged columns: (stage column << 11) | (shift << 6) | width.
// Aggregation descriptor of one query (32 bytes, shared memory). The group index is
// k0*kmul0 + k1*kmul1 + bias in 32-bit wrapping arithmetic, which equals
// (k0 - kmin0)*kmul0 + (k1 - kmin1)*kmul1 with bias = -(kmin0*kmul0 + kmin1*kmul1); an
// absent key has multiplier 0. Scalars are one-group arrays.
struct __align__(16) AQ {
  uint16_t a0, a1, k0, k1;  // stage field codes
  unsigned kmul0, kmul1, bias;
  int total;                // groups (1 for a scalar)
  int soff;                 // shared-memory byte offset of the 64-bit sums; < 0: sums by L2
                            // atomics, and soff <= -2 puts the keys' touch bitmap at -soff - 2
  int flags;                // bits 0-1 agg op, bit 2 CRYSTAL4 keys, bits 3-4 number of keys,
                            // bit 5 a scalar kept in kScalarCopies words (lane mod 4 adds to
                            // its own), bits 8-16 its family's group stride, bits 17-25 its
                            // place in it
};
// A family is a set of queries with the same group count whose shared-memory sums are
// interleaved group-major: the sum of group g of the family's j-th query lies at
// base + 8 * (g * stride + j) (soff = base + 8 * j), so the matches of one row — same
// group, neighbouring queries — hit neighbouring words rather than banks at random. The
// stride is the member count rounded up to an odd number: matches of one query to
// different groups (rows of one date on a date-sorted table match the same queries) then
// fall in different bank pairs, where an even stride that is a multiple of 16 would put
// them all in one. The members' touch bitmaps follow the sums:
// base + 8 * total * stride + 4 * words * j. A query alone is a family of one.
__device__ __forceinline__ int aq_family(const AQ& A) { return (A.flags >> 8) & 0x1ff; }
__device__ __forceinline__ int aq_member(const AQ& A) { return (A.flags >> 17) & 0x1ff; }
static_assert(sizeof(AQ) == 32, "aggregation descriptor size");

// Per-query descriptor in the launch parameters (96 bytes).
struct BQ {
  AQ a;
  uint8_t np, res_layout, pad[2];
  uint16_t pf[MB_BATCH_MAX_PREDS];  // row-schema field codes of the predicates
  int plo[MB_BATCH_MAX_PREDS], phi[MB_BATCH_MAX_PREDS];
  int pad2;
  void* res;
};
static_assert(sizeof(BQ) == 96, "descriptor size");

struct BatchPlan {
  long long n, nfull;
  int ncols;                       // staged fact columns
  const int* col[MB_NUM_FACT_COLS];
  int cidx[13];                    // row-schema column -> stage column (-1: absent)
  int stage_dim[kMaxStageCols];    // stage column -> dimension whose word it holds (-1: fact column)
  int ndims;
  int dim_list[4];
  int key_stage[4];
  const unsigned* pat[4];
  int pat_slots[4], pat_kmin[4];
  int nq, nwords;
  int nfields;                     // attributes some query constrains
  int f_code[kMaxPredFields], f_scode[kMaxPredFields], f_min[kMaxPredFields], f_n[kMaxPredFields];
  int f_smem_off[kMaxPredFields];  // byte offset of the table in shared memory, -1: workspace
  long long f_goff[kMaxPredFields];// word offset of the table in the workspace
  int f_ent[kMaxPredFields];       // table entries: f_n, or f_nint for an interval-coded attribute
  // Interval coding of a wide attribute (hull wider than kSmemTableMaxEntries values): the
  // queries' range end points cut the hull into f_nint intervals on which every query's
  // verdict is constant; the table holds one mask per interval. A value v (relative to
  // f_min) is in interval i when bp[i] <= v < bp[i+1]; bucket v >> f_shift of a shared-
  // memory index gives the interval of the bucket's first value, and a short forward
  // scan over the end points finishes the search.
  int f_nint[kMaxPredFields], f_bp_off[kMaxPredFields], f_shift[kMaxPredFields];
  int f_bps_off[kMaxPredFields], f_bkt_off[kMaxPredFields];  // shared-memory byte offsets
  int bp[kMaxBreakpoints];
  unsigned outside[kMaxPredFields][kMaskWordsMax];  // mask for values outside the hull
  unsigned pres_mask[16][kMaskWordsMax];
  unsigned* tables;                // workspace
  long long table_entries;
  int stages, stage_words, list_cap;
  int smem_acc_off, smem_aq_off, smem_res_off, smem_pres_off, smem_out_off, smem_list_off;
  int acc_words;                   // 8-byte scalar words (kScalarCopies per scalar query)
  int smem_groups_off, smem_groups_words, smem_stage_off;
  unsigned int* status;
  // segment-cache addressing: col[c] is a per-segment slot array into gpu_cache
  const int* gpu_cache;
  const short* seg_group;
  int seg_shift;
  BQ q[MB_BATCH_MAX_QUERIES];
};
static_assert(sizeof(BatchPlan) < 32000, "launch parameter limit");

__device__ __forceinline__ int bslot(int key, int slots, int kmin) {
  const int d = static_cast<int>(static_cast<unsigned>(key) - static_cast<unsigned>(kmin));
  if (static_cast<unsigned>(d) < static_cast<unsigned>(slots)) return d;
  if (static_cast<unsigned>(d) < 2u * static_cast<unsigned>(slots)) return d - slots;
  return d % slots;
}

// Physical tile of scan position t (CTA b takes positions b, b + G, b + 2G, ...). The
// first kTileRegions * Q tiles (Q = nfull / kTileRegions) are visited column-major over
// kTileRegions regions of the table, so the tiles the grid holds at one moment lie in
// different regions rather than side by side. On a table sorted by date, side-by-side
// tiles share a date: every SM would then add into the same queries' group records (the
// same year's) at once, while the regions spread those updates over the table's years.
// Every CTA still sees every region, so the work stays balanced.
constexpr long long kTileRegions = 16;
__device__ __forceinline__ long long tile_order(long long t, long long nfull) {
  const long long q = nfull / kTileRegions;
  if (t >= q * kTileRegions) return t;
  return (t % kTileRegions) * q + t / kTileRegions;
}

__device__ __forceinline__ int field_value(int v, int code) {
  const int width = code & 63;
  const unsigned shift = (code >> 6) & 31;
  const unsigned mask = width >= 32 ? 0xffffffffu : (1u << width) - 1u;
  return static_cast<int>((static_cast<unsigned>(v) >> shift) & mask);
}

// Stage column c, row r, read from global memory (direct, or through the segment cache).
__device__ __forceinline__ int batch_load(const BatchPlan& P, int c, long long r) {
  if (P.gpu_cache == nullptr) return __ldg(P.col[c] + r);
  const long long vseg = r >> P.seg_shift;
  const int seg = P.seg_group ? static_cast<int>(P.seg_group[vseg]) : static_cast<int>(vseg);
  return __ldg(P.gpu_cache + (static_cast<long long>(__ldg(P.col[c] + seg)) << P.seg_shift) +
               (r & ((1ll << P.seg_shift) - 1)));
}

__device__ __forceinline__ void bmbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ AQ load_aq(const AQ* s_aq, int qi) {
  const uint4* p = reinterpret_cast<const uint4*>(s_aq + qi);
  const uint4 x = p[0], y = p[1];
  AQ a;
  a.a0 = static_cast<uint16_t>(x.x);
  a.a1 = static_cast<uint16_t>(x.x >> 16);
  a.k0 = static_cast<uint16_t>(x.y);
  a.k1 = static_cast<uint16_t>(x.y >> 16);
  a.kmul0 = x.z;
  a.kmul1 = x.w;
  a.bias = y.x;
  a.total = static_cast<int>(y.y);
  a.soff = static_cast<int>(y.z);
  a.flags = static_cast<int>(y.w);
  return a;
}

// The 32-bit value a match adds (sign-extended to 64 bits by the caller), as the
// single-query path computes it: SUM a0, SUB a0 - a1, MUL a0 * a1 (wrapping).
template <class Get>
__device__ __forceinline__ unsigned batch_value(const AQ& A, Get get) {
  const unsigned v0 = static_cast<unsigned>(get(A.a0)), v1 = static_cast<unsigned>(get(A.a1));
  const int op = A.flags & 3;
  return op == MB_AGG_SUM ? v0 : op == MB_AGG_SUB ? v0 - v1 : v0 * v1;
}

// Add one (row, query) match: `get(code)` reads a field of the row.
template <class Get>
__device__ __forceinline__ void batch_match(const AQ& A, void* const* s_res, int qi, Get get, unsigned char* smem,
                                            bool& bad_group) {
  const unsigned u = batch_value(A, get);
  const unsigned long long w = static_cast<unsigned long long>(static_cast<long long>(static_cast<int>(u)));
  const int k0 = get(A.k0), k1 = get(A.k1);
  const unsigned hh = static_cast<unsigned>(k0) * A.kmul0 + static_cast<unsigned>(k1) * A.kmul1 + A.bias;
  int g = static_cast<int>(hh);
  if (hh >= static_cast<unsigned>(A.total)) {
    g %= A.total;
    if (g < 0) {
      bad_group = true;
      return;
    }
  }
  const bool c4 = (A.flags >> 2) & 1;
  if (A.soff >= 0) {
    const int fam = aq_family(A), j = aq_member(A);
    const int copy = (A.flags >> 5) & 1 ? static_cast<int>(threadIdx.x & (kScalarCopies - 1)) : 0;
    atomicAdd(reinterpret_cast<unsigned long long*>(smem + A.soff) + g * fam + copy, w);
    if (!c4) return;
    // the first row of a group in this CTA writes the group's keys
    uint32_t* s_touch = reinterpret_cast<uint32_t*>(smem + A.soff - 8 * j + 8 * A.total * fam) +
                        j * ((A.total + 31) >> 5);
    const uint32_t bit = 1u << (g & 31);
    if ((s_touch[g >> 5] & bit) || (atomicOr(&s_touch[g >> 5], bit) & bit)) return;
  } else {
    void* res = s_res[qi];
    atomicAdd(c4 ? reinterpret_cast<unsigned long long*>(static_cast<int*>(res) + 4 * g + 2)
                 : static_cast<unsigned long long*>(res) + g,
              w);
    if (!c4) return;
    if (A.soff <= -2) {
      // keys once per CTA and group: the group records are few lines that every SM updates
      uint32_t* s_touch = reinterpret_cast<uint32_t*>(smem + (-A.soff - 2));
      const uint32_t bit = 1u << (g & 31);
      if ((s_touch[g >> 5] & bit) || (atomicOr(&s_touch[g >> 5], bit) & bit)) return;
    }
  }
  int* res = static_cast<int*>(s_res[qi]);
  const int nk = (A.flags >> 3) & 3;
  if (nk > 1)
    *reinterpret_cast<int2*>(res + 4 * g) = make_int2(k0, k1);  // one 8-byte store (16-byte records)
  else if (nk > 0)
    res[4 * g] = k0;
}

// The queries accepting one row: presence mask AND one mask per constrained attribute.
// `get(code)` reads a field of the row.
template <int NWM, class Get>
__device__ __forceinline__ void batch_row_mask(const BatchPlan& P, unsigned pres, Get get, const unsigned* s_pres,
                                               const unsigned* s_out, const unsigned char* smem, unsigned (&m)[NWM]) {
#pragma unroll
  for (int w = 0; w < NWM; ++w) m[w] = s_pres[pres * kMaskWordsMax + w];
#pragma unroll
  for (int f = 0; f < kMaxPredFields; ++f) {
    if (f >= P.nfields) break;
    // with one mask word an empty mask ends the row early; with more, rows nearly always
    // keep some query and the test would cost more than it saves
    if (NWM == 1 && m[0] == 0) return;
    const int v = get(P.f_scode[f]) - P.f_min[f];
    const unsigned* t;
    if (static_cast<unsigned>(v) < static_cast<unsigned>(P.f_n[f])) {
      int e = v;
      if (P.f_nint[f] > 0) {
        const int* bp = reinterpret_cast<const int*>(smem + P.f_bps_off[f]);
        e = reinterpret_cast<const uint16_t*>(smem + P.f_bkt_off[f])[v >> P.f_shift[f]];
        while (e + 1 < P.f_nint[f] && bp[e + 1] <= v) ++e;
      }
      t = P.f_smem_off[f] >= 0 ? reinterpret_cast<const unsigned*>(smem + P.f_smem_off[f]) + e * P.nwords
                               : P.tables + P.f_goff[f] + static_cast<long long>(e) * P.nwords;
    } else
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

template <int NCW, int ITEMS, int NWM>
__global__ void __launch_bounds__((NCW + 1) * 32, 1) batch_kernel(const __grid_constant__ BatchPlan P) {
  constexpr int WROWS = 32 * ITEMS;
  constexpr int TILE = NCW * WROWS;
  constexpr int CS = TILE + kColPad;  // stage column stride (words)
  constexpr int NWARPS = NCW + 1;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kBatchStages;
  AQ* s_aq = reinterpret_cast<AQ*>(smem + P.smem_aq_off);
  void** s_res = reinterpret_cast<void**>(smem + P.smem_res_off);
  unsigned* s_pres = reinterpret_cast<unsigned*>(smem + P.smem_pres_off);
  unsigned* s_out = reinterpret_cast<unsigned*>(smem + P.smem_out_off);
  int* stage_base = reinterpret_cast<int*>(smem + P.smem_stage_off);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = P.stages;

  // ---- set-up: accumulators, descriptors, masks, small tables, barriers ------------
  {
    unsigned long long* s_acc = reinterpret_cast<unsigned long long*>(smem + P.smem_acc_off);
    for (int w = tid; w < P.acc_words; w += NWARPS * 32) s_acc[w] = 0;
    for (int q = tid; q < P.nq; q += NWARPS * 32) s_res[q] = P.q[q].res;
    unsigned* dst = reinterpret_cast<unsigned*>(s_aq);
    for (int w = tid; w < P.nq * 8; w += NWARPS * 32) dst[w] = reinterpret_cast<const unsigned*>(&P.q[w >> 3].a)[w & 7];
    for (int w = tid; w < 16 * kMaskWordsMax; w += NWARPS * 32) s_pres[w] = (&P.pres_mask[0][0])[w];
    for (int w = tid; w < kMaxPredFields * kMaskWordsMax; w += NWARPS * 32) s_out[w] = (&P.outside[0][0])[w];
    unsigned* g = reinterpret_cast<unsigned*>(smem + P.smem_groups_off);
    for (int w = tid; w < P.smem_groups_words; w += NWARPS * 32) g[w] = 0;
    for (int f = 0; f < P.nfields; ++f) {
      if (P.f_smem_off[f] < 0) continue;
      unsigned* t = reinterpret_cast<unsigned*>(smem + P.f_smem_off[f]);
      const unsigned* s = P.tables + P.f_goff[f];
      for (int w = tid; w < P.f_ent[f] * P.nwords; w += NWARPS * 32) t[w] = s[w];
      if (P.f_nint[f] > 0) {
        int* bp = reinterpret_cast<int*>(smem + P.f_bps_off[f]);
        for (int i = tid; i < P.f_nint[f]; i += NWARPS * 32) bp[i] = P.bp[P.f_bp_off[f] + i];
      }
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
  // bucket indexes of the interval-coded attributes: the interval of each bucket's first value
  for (int f = 0; f < P.nfields; ++f) {
    if (P.f_nint[f] == 0) continue;
    const int* bp = reinterpret_cast<const int*>(smem + P.f_bps_off[f]);
    uint16_t* bkt = reinterpret_cast<uint16_t*>(smem + P.f_bkt_off[f]);
    const int nb = ((P.f_n[f] - 1) >> P.f_shift[f]) + 1;
    for (int b = tid; b < nb; b += NWARPS * 32) {
      const int v0 = b << P.f_shift[f];
      int lo = 0, hi = P.f_nint[f] - 1;  // bp[0] = 0 <= v0: find the last bp[i] <= v0
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bp[mid] <= v0)
          lo = mid;
        else
          hi = mid - 1;
      }
      bkt[b] = static_cast<uint16_t>(lo);
    }
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
        const long long r0 = tile_order(b + k * G, P.nfull) * static_cast<long long>(TILE);
        int* dst = stage_base + s * P.stage_words;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>(P.ncols) * TILE * 4u);
        if (P.gpu_cache == nullptr) {
          for (int c = 0; c < P.ncols; ++c) bulk_g2s(dst + c * CS, P.col[c] + r0, TILE * 4, &full[s], policy);
        } else {
          // through the segment cache: a tile that crosses a segment boundary is copied in
          // two pieces (row offsets are multiples of 4, so every piece is 16-byte aligned)
          const long long S = 1ll << P.seg_shift;
          for (int done = 0; done < TILE;) {
            const long long r = r0 + done;
            const long long vseg = r >> P.seg_shift;
            const int seg = P.seg_group ? static_cast<int>(P.seg_group[vseg]) : static_cast<int>(vseg);
            const long long in = r & (S - 1);
            const int take = static_cast<int>(S - in < TILE - done ? S - in : TILE - done);
            // all slots first (their loads in flight together), then the ordered copies
            int slot[MB_NUM_FACT_COLS];
#pragma unroll
            for (int c = 0; c < MB_NUM_FACT_COLS; ++c)
              if (c < P.ncols) slot[c] = P.col[c][seg];
#pragma unroll
            for (int c = 0; c < MB_NUM_FACT_COLS; ++c)
              if (c < P.ncols)
                bulk_g2s(dst + c * CS + done, P.gpu_cache + (static_cast<long long>(slot[c]) << P.seg_shift) + in,
                         static_cast<uint32_t>(take) * 4u, &full[s], policy);
            done += take;
          }
        }
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
    unsigned* mlist = reinterpret_cast<unsigned*>(smem + P.smem_list_off) + cw * P.list_cap;
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
        const int* kcol = wst + P.key_stage[d] * CS;
        int* out = wst + P.cidx[MB_COL_DIM_S + d] * CS;
        const unsigned* pat = P.pat[d];
        const int slots = P.pat_slots[d], kmin = P.pat_kmin[d];
        unsigned wv[ITEMS];
        auto lookup = [&](int key) -> unsigned {
          const int h = bslot(key, slots, kmin);
          if (h < 0) {
            bad_probe = true;
            return 0u;
          }
          return __ldg(pat + h);
        };
        if constexpr (ITEMS % 4 == 0) {
#pragma unroll
          for (int j = 0; j < ITEMS / 4; ++j) {
            const int4 kv = lds128(kcol + (j * 32 + lane) * 4);
            wv[4 * j] = lookup(kv.x);
            wv[4 * j + 1] = lookup(kv.y);
            wv[4 * j + 2] = lookup(kv.z);
            wv[4 * j + 3] = lookup(kv.w);
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
        } else {
#pragma unroll
          for (int e = 0; e < ITEMS; ++e) wv[e] = lookup(kcol[e * 32 + lane]);
#pragma unroll
          for (int e = 0; e < ITEMS; ++e) out[e * 32 + lane] = static_cast<int>(wv[e]);
        }
      }
      __syncwarp();
      // ---- query masks row by row (lane l takes rows l, 32 + l, ...); matches go
      // through the warp's list so that every lane aggregates one pair at a time ------
      int lpos = 0;
      auto flush = [&](int n) {
        for (int base = 0; base < n; base += 32) {
          const int idx = base + lane;
          if (idx < n) {
            const unsigned pr = mlist[idx];
            const int row = static_cast<int>(pr >> 16), qi = static_cast<int>(pr & 0xffffu);
            auto get = [&](int code) { return field_value(wst[(code >> 11) * CS + row], code); };
            batch_match(load_aq(s_aq, qi), s_res, qi, get, smem, bad_group);
          }
        }
        __syncwarp();
      };
#pragma unroll 1
      for (int i = 0; i < ITEMS; ++i) {
        const int row = i * 32 + lane;
        unsigned pres = 0;
        for (int t = 0; t < P.ndims; ++t) {
          const int d = P.dim_list[t];
          pres |= (static_cast<unsigned>(wst[P.cidx[MB_COL_DIM_S + d] * CS + row]) >> 31) << d;
        }
        auto get = [&](int code) { return field_value(wst[(code >> 11) * CS + row], code); };
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
        if (lpos + total > P.list_cap) {
          flush(lpos);
          lpos = 0;
        }
        if (total > P.list_cap) {
          // more matches than the list holds: this row runs lane by lane
#pragma unroll
          for (int w = 0; w < NWM; ++w) {
            unsigned bits = m[w];
            while (bits) {
              const int qi = w * 32 + __ffs(bits) - 1;
              bits &= bits - 1;
              batch_match(load_aq(s_aq, qi), s_res, qi, get, smem, bad_group);
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
          const int h = bslot(batch_load(P, P.key_stage[d], r), P.pat_slots[d], P.pat_kmin[d]);
          if (h < 0) {
            bad_probe = true;
            continue;
          }
          dimw[d] = static_cast<int>(__ldg(P.pat[d] + h));
          pr |= (static_cast<unsigned>(dimw[d]) >> 31) << d;
        }
        auto get = [&](int code) {
          const int c = code >> 11;
          const int d = P.stage_dim[c];
          return field_value(d >= 0 ? dimw[d] : batch_load(P, c, r), code);
        };
        unsigned m[NWM];
        batch_row_mask<NWM>(P, pr, get, s_pres, s_out, smem, m);
#pragma unroll
        for (int w = 0; w < NWM; ++w) {
          unsigned bits = m[w];
          while (bits) {
            const int qi = w * 32 + __ffs(bits) - 1;
            bits &= bits - 1;
            batch_match(load_aq(s_aq, qi), s_res, qi, get, smem, bad_group);
          }
        }
      }
    }
  }

  if (failed) set_status(P.status, MB_STATUS_TIMEOUT);
  if (bad_probe) set_status(P.status, MB_STATUS_PROBE_RANGE);
  if (bad_group) set_status(P.status, MB_STATUS_GROUP_RANGE);
  __syncthreads();
  // ---- fold this CTA's scalars and shared-memory group arrays into the results -------
  // (a zero partial is skipped: adding it changes nothing)
  for (int q = 0; q < P.nq; ++q) {
    const AQ A = s_aq[q];
    if (A.soff < 0) continue;
    const unsigned long long* s_sum = reinterpret_cast<const unsigned long long*>(smem + A.soff);
    const bool c4 = (A.flags >> 2) & 1;
    const int fam = aq_family(A);
    const bool copies = (A.flags >> 5) & 1;
    for (int g = tid; g < A.total; g += NWARPS * 32) {
      unsigned long long v = s_sum[g * fam];
      if (copies)
        for (int k = 1; k < kScalarCopies; ++k) v += s_sum[k];
      if (v == 0) continue;
      atomicAdd(c4 ? reinterpret_cast<unsigned long long*>(static_cast<int*>(s_res[q]) + 4 * g + 2)
                   : static_cast<unsigned long long*>(s_res[q]) + g,
                v);
    }
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
    while (f < P.nfields - 1 && v >= P.f_ent[f]) v -= P.f_ent[f++];
    // an interval's verdicts are those of its first value
    const int x = P.f_min[f] + (P.f_nint[f] > 0 ? P.bp[P.f_bp_off[f] + v] : static_cast<int>(v));
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
// (consumer warps, rows per lane per stage): more warps per CTA hide more latency; fewer
// rows per lane keep their stage ring small enough for that
static const BatchVariant kBatchVariants[] = {
    MB_BATCH_VARIANTS(8, 4), MB_BATCH_VARIANTS(16, 4), MB_BATCH_VARIANTS(16, 2),
    MB_BATCH_VARIANTS(24, 1), MB_BATCH_VARIANTS(24, 2), MB_BATCH_VARIANTS(30, 1),
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
  // row-schema codes of the aggregation fields, converted to stage codes below
  int af[MB_BATCH_MAX_QUERIES][2], kf[MB_BATCH_MAX_QUERIES][2];
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
    const int nk = q.res_layout == MB_RES_SCALAR ? 0 : q.num_keys;
    d.np = static_cast<uint8_t>(q.num_preds);
    d.res_layout = static_cast<uint8_t>(q.res_layout);
    dims_used |= static_cast<unsigned>(q.dims_required);
    for (int p = 0; p < q.num_preds; ++p) {
      if (!note_field(q.pred_field[p])) return MB_ERR_ARG;
      d.pf[p] = static_cast<uint16_t>(q.pred_field[p]);
      d.plo[p] = q.pred_lo[p];
      d.phi[p] = q.pred_hi[p];
    }
    for (int k = 0; k < (q.agg_op == MB_AGG_SUM ? 1 : 2); ++k)
      if (!note_field(q.agg_field[k])) return MB_ERR_ARG;
    af[qi][0] = q.agg_field[0];
    af[qi][1] = q.agg_op == MB_AGG_SUM ? q.agg_field[0] : q.agg_field[1];
    for (int k = 0; k < nk; ++k)
      if (!note_field(q.key_field[k])) return MB_ERR_ARG;
    // an absent key reads the first aggregation field and weighs it by 0
    kf[qi][0] = nk > 0 ? q.key_field[0] : af[qi][0];
    kf[qi][1] = nk > 1 ? q.key_field[1] : af[qi][0];
    AQ& A = d.a;
    A.kmul0 = nk > 0 ? static_cast<unsigned>(q.key_mul[0]) : 0u;
    A.kmul1 = nk > 1 ? static_cast<unsigned>(q.key_mul[1]) : 0u;
    A.bias = 0u - ((nk > 0 ? static_cast<unsigned>(q.key_min[0]) * A.kmul0 : 0u) +
                   (nk > 1 ? static_cast<unsigned>(q.key_min[1]) * A.kmul1 : 0u));
    A.total = q.res_layout == MB_RES_SCALAR ? 1 : q.total_val;
    A.soff = -1;
    A.flags = q.agg_op | ((q.res_layout == MB_RES_CRYSTAL4 ? 1 : 0) << 2) | (nk << 3) | (1 << 8);
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
  int nbp = 0;
  for (int f = 0; f < P.nfields; ++f) {
    const long long n = has[f] ? static_cast<long long>(hmax[f]) - hmin[f] + 1 : 1;
    if (n > 65536) return MB_ERR_SIZE;  // attribute ranges wider than 65,536 values
    P.f_min[f] = has[f] ? hmin[f] : 0;
    P.f_n[f] = static_cast<int>(n);
    P.f_ent[f] = P.f_n[f];
    if (n > kSmemTableMaxEntries) {
      // interval coding: end points lo and hi + 1 of every non-empty range on f, and 0
      int pts[2 * MB_BATCH_MAX_QUERIES * MB_BATCH_MAX_PREDS + 1];
      int np = 0;
      pts[np++] = 0;
      for (int qi = 0; qi < P.nq; ++qi) {
        const BQ& d = P.q[qi];
        for (int p = 0; p < d.np; ++p) {
          if (d.pf[p] != P.f_code[f] || d.plo[p] > d.phi[p]) continue;
          const long long lo = static_cast<long long>(d.plo[p]) - P.f_min[f];
          const long long hi1 = static_cast<long long>(d.phi[p]) + 1 - P.f_min[f];
          if (lo > 0) pts[np++] = static_cast<int>(lo);
          if (hi1 < n) pts[np++] = static_cast<int>(hi1);
        }
      }
      std::sort(pts, pts + np);
      np = static_cast<int>(std::unique(pts, pts + np) - pts);
      if (nbp + np <= kMaxBreakpoints) {
        P.f_nint[f] = np;
        P.f_bp_off[f] = nbp;
        for (int i = 0; i < np; ++i) P.bp[nbp + i] = pts[i];
        nbp += np;
        int shift = 0;
        while ((static_cast<long long>(kMaxBuckets) << shift) < n) ++shift;
        P.f_shift[f] = shift;
        P.f_ent[f] = np;
      }
    }
    P.f_goff[f] = entries * P.nwords;
    entries += P.f_ent[f];
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
    for (int qi = 0; qi < P.nq; ++qi) {
      const unsigned req = static_cast<unsigned>(a->queries[qi].dims_required);
      if ((pm & req) == req) P.pres_mask[pm][qi / 32] |= 1u << (qi % 32);
    }

  // dimensions: their keys are staged, their words overwrite the key columns (the date
  // word gets its own column because orderdate is also a field)
  static const int kKeyCol[4] = {MB_COL_SUPPKEY, MB_COL_CUSTKEY, MB_COL_PARTKEY, MB_COL_ORDERDATE};
  for (int d = 0; d < 4; ++d) {
    if (!(dims_used & (1u << d))) continue;
    if (a->dim[d].words == nullptr || a->dim[d].slots <= 0 || a->fact[kKeyCol[d]] == nullptr) return MB_ERR_ARG;
    fact_used[kKeyCol[d]] = true;
  }
  for (int c = 0; c < 13; ++c) P.cidx[c] = -1;
  for (int c = 0; c < kMaxStageCols; ++c) P.stage_dim[c] = -1;
  if (a->gpu_cache != nullptr) {
    const int ss = a->segment_size;
    if (ss < 4 || (ss & (ss - 1)) != 0) return MB_ERR_ARG;
    if (!aligned16(a->gpu_cache)) return MB_ERR_ALIGN;
    P.gpu_cache = a->gpu_cache;
    P.seg_group = a->segment_group;
    P.seg_shift = __builtin_ctz(static_cast<unsigned>(ss));
  } else if (a->segment_group != nullptr) {
    return MB_ERR_ARG;
  }
  for (int c = 0; c < MB_NUM_FACT_COLS; ++c) {
    if (!fact_used[c]) continue;
    if (P.gpu_cache == nullptr && !aligned16(a->fact[c])) return MB_ERR_ALIGN;
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
    P.stage_dim[P.cidx[MB_COL_DIM_S + d]] = d;
  }
  // a dimension word that replaces its key makes that key unavailable as a field
  auto uses_key = [&](int code) {
    const int col = code >> 11;
    for (int t = 0; t < 3; ++t)
      if ((dims_used & (1u << t)) && col == kKeyCol[t]) return true;
    return false;
  };
  for (int qi = 0; qi < P.nq; ++qi) {
    const BQ& d = P.q[qi];
    for (int p = 0; p < d.np; ++p)
      if (uses_key(d.pf[p])) return MB_ERR_ARG;
    for (int k = 0; k < 2; ++k)
      if (uses_key(af[qi][k]) || uses_key(kf[qi][k])) return MB_ERR_ARG;
  }
  // stage codes
  auto scode = [&](int code) { return (P.cidx[code >> 11] << 11) | (code & 0x7ff); };
  for (int f = 0; f < P.nfields; ++f) P.f_scode[f] = scode(P.f_code[f]);
  for (int qi = 0; qi < P.nq; ++qi) {
    AQ& A = P.q[qi].a;
    A.a0 = static_cast<uint16_t>(scode(af[qi][0]));
    A.a1 = static_cast<uint16_t>(scode(af[qi][1]));
    A.k0 = static_cast<uint16_t>(scode(kf[qi][0]));
    A.k1 = static_cast<uint16_t>(scode(kf[qi][1]));
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

  // defaults measured best for 256 queries over 120M rows: 24 consumer warps, one row a lane
  const int threads = a->threads ? a->threads : 768;
  const int items = a->items_per_thread ? a->items_per_thread : 1;
  const int nwm = P.nwords;
  const BatchVariant* var = nullptr;
  for (const BatchVariant& v : kBatchVariants)
    if (v.warps * 32 == threads && v.items == items && v.nwm == nwm) var = &v;
  if (var == nullptr) return MB_ERR_ARG;
  const int tile = threads * items;
  P.nfull = P.n / tile;
  P.stage_words = (P.ncols + ((P.ndims && P.dim_list[P.ndims - 1] == 3) ? 1 : 0)) * (tile + kColPad);
  int stages = a->stages ? a->stages : 2;
  if (stages < 2 || stages > kBatchStages) return MB_ERR_ARG;

  // shared memory: barriers | scalars | aggregation descriptors | result pointers |
  // presence masks | outside masks | small predicate tables | match lists |
  // small group arrays | stage ring
  int off = 2 * kBatchStages * 8;
  int nscalar = 0;
  for (int qi = 0; qi < P.nq; ++qi) nscalar += P.q[qi].res_layout == MB_RES_SCALAR ? 1 : 0;
  P.smem_acc_off = off;
  P.acc_words = kScalarCopies * nscalar;
  off += 8 * P.acc_words;
  off = (off + 15) / 16 * 16;
  P.smem_aq_off = off;
  off += static_cast<int>(sizeof(AQ)) * P.nq;
  P.smem_res_off = off;
  off += 8 * P.nq;
  off = (off + 15) / 16 * 16;
  P.smem_pres_off = off;
  off += 16 * kMaskWordsMax * 4;
  P.smem_out_off = off;
  off += kMaxPredFields * kMaskWordsMax * 4;
  for (int f = 0; f < P.nfields; ++f) {
    P.f_smem_off[f] = -1;
    if (P.f_ent[f] <= kSmemTableMaxEntries || P.f_nint[f] > 0) {
      P.f_smem_off[f] = off;
      off += (P.f_ent[f] * P.nwords * 4 + 15) / 16 * 16;
    }
    if (P.f_nint[f] > 0) {
      P.f_bps_off[f] = off;
      off += (P.f_nint[f] * 4 + 15) / 16 * 16;
      P.f_bkt_off[f] = off;
      off += ((((P.f_n[f] - 1) >> P.f_shift[f]) + 1) * 2 + 15) / 16 * 16;
    }
  }
  P.smem_list_off = off;
  const int budget = ds->max_smem_optin - 2048;
  auto total_smem = [&](int base, int st) { return (base + 127) / 128 * 128 + st * P.stage_words * 4; };
  // match lists: 1,024 pairs a warp, or 512 where that leaves shared-memory group arrays
  // less than 64 KB (a list must hold the pairs of 32 rows with ease: ~8 queries a row
  // pass on average in a batch of 256 with log-uniform selectivities up to 0.3)
  P.list_cap = kMatchListMax;
  if (total_smem(off + (threads / 32) * P.list_cap * 4, stages) > budget - 65536) P.list_cap = 512;
  off += (threads / 32) * P.list_cap * 4;
  while (total_smem(off, stages) > budget && stages > 2) --stages;
  if (total_smem(off, stages) > budget) return MB_ERR_SIZE;
  P.stages = stages;
  // scalars accumulate in their shared-memory words (kScalarCopies each)
  for (int qi = 0, k = 0; qi < P.nq; ++qi)
    if (P.q[qi].res_layout == MB_RES_SCALAR) {
      P.q[qi].a.soff = P.smem_acc_off + 8 * kScalarCopies * k++;
      P.q[qi].a.flags |= 1 << 5;
    }
  // small group arrays (<= 1,024 groups) to shared memory, smallest first, within the budget
  P.smem_groups_off = off;
  int groups_bytes = 0;
  const int group_cap = a->smem_group_bytes < 0 ? 131072 : a->smem_group_bytes;
  // shared memory kept for the touch bitmaps of the small-array queries that end up with
  // L2 sums (below): a few bytes each, and without one such a query writes its keys on
  // every match
  int touch_reserve = 0;
  for (int qi = 0; qi < P.nq; ++qi) {
    const AQ& A = P.q[qi].a;
    if (P.q[qi].res_layout != MB_RES_SCALAR && ((A.flags >> 2) & 1) && A.total <= 1024)
      touch_reserve += (4 * ((A.total + 31) / 32) + 15) / 16 * 16;
  }
  // queries with the same group count form a family (group-major interleaved sums); as
  // many members as fit, smallest group counts first
  for (;;) {
    int total = 0;
    for (int qi = 0; qi < P.nq; ++qi) {
      const AQ& A = P.q[qi].a;
      if (P.q[qi].res_layout == MB_RES_SCALAR || A.soff >= 0 || A.total > 1024 || (A.flags & (1 << 30))) continue;
      if (total == 0 || A.total < total) total = A.total;
    }
    if (total == 0) break;
    const int words = (total + 31) / 32;
    auto fam_bytes = [&](int k) { return (8 * total * (k | 1) + 4 * words * k + 15) / 16 * 16; };
    int members = 0;
    for (int qi = 0; qi < P.nq; ++qi) {
      const AQ& A = P.q[qi].a;
      if (P.q[qi].res_layout == MB_RES_SCALAR || A.soff >= 0 || A.total != total) continue;
      if (groups_bytes + fam_bytes(members + 1) > group_cap ||
          total_smem(off + groups_bytes + fam_bytes(members + 1) + touch_reserve, stages) > budget)
        break;
      ++members;
    }
    int j = 0;
    for (int qi = 0; qi < P.nq; ++qi) {
      AQ& A = P.q[qi].a;
      if (P.q[qi].res_layout == MB_RES_SCALAR || A.soff >= 0 || A.total != total) continue;
      if (j < members) {
        A.soff = off + groups_bytes + 8 * j;
        A.flags = (A.flags & 0xff) | ((members | 1) << 8) | (j << 17);
        ++j;
      } else {
        A.flags |= 1 << 30;  // no room: sums by L2 atomics (marked so the search moves on)
      }
    }
    groups_bytes += fam_bytes(members);
  }
  for (int qi = 0; qi < P.nq; ++qi) P.q[qi].a.flags &= ~(1 << 30);
  // queries left with L2 sums that write keys, and few groups (a few hot result lines),
  // get a touch bitmap in shared memory where it fits (smallest group counts first), so
  // they write their keys once per CTA and group; with many groups the stores spread out
  // and cost less than the test
  for (int pass_total = 1; pass_total <= 1024; pass_total *= 2) {
    for (int qi = 0; qi < P.nq; ++qi) {
      AQ& A = P.q[qi].a;
      if (A.soff != -1 || !((A.flags >> 2) & 1) || A.total > pass_total || A.total <= pass_total / 2) continue;
      const int bytes = (4 * ((A.total + 31) / 32) + 15) / 16 * 16;
      if (total_smem(off + groups_bytes + bytes, stages) > budget) continue;
      A.soff = -(off + groups_bytes) - 2;
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
