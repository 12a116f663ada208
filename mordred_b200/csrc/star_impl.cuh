// star_impl.cuh — device code of the fused star-query kernel (see star.cuh), shared by
// the translation units that instantiate its variants.
//
// Semantics follow the reference kernels row for row:
//   filters      GPUProcessing.h:74-86 (fact BETWEEN), crystal/pred.cuh (EQ, EQ OR EQ)
//   probes       crystal/join.cuh:5-165 (PHT_1 / PHT_2), BlockLibrary.cuh:86-111 (engine)
//   group index  GPUProcessing.h:143 ((g1-m1)*u1 + ... ) % total_val, int32 arithmetic
//   aggregate    q11.cu:74 (int32 product widened), GPUProcessing.h:149-150 (int32 difference)
// Rows are independent and every sum is a 64-bit integer, so the order in which tiles,
// rows and atomics are applied cannot change any result bit.
#pragma once

#include "star.cuh"

namespace mb {

constexpr unsigned kFull = 0xffffffffu;

// A compiled kernel variant: consumer warps, rows per lane per tile and the query
// shape it is specialised for (-1 = read from the plan at run time).
using KernelFn = void (*)(StarPlan);
struct Variant {
  int warps, items, nf, nd, ns;
  KernelFn fn;
  bool mir = false;   // reads cluster-resident mirrors (launched with a cluster)
  bool pack = false;  // packs the first sparse probe's survivors across the warp
  bool rel = false;   // returns each stage before its last batch's probes (columns in registers)
};

__device__ __forceinline__ bool pass_filter(int x, int mode, int c1, int c2) {
  if (mode == MB_FILTER_BETWEEN) return x >= c1 && x <= c2;
  if (mode == MB_FILTER_EQ) return x == c1;
  return x == c1 || x == c2;
}

// Out-of-line remainder for the rare keys outside [key_min, key_min + 2*slots): kept as
// a call so the hot path never carries an if-converted division.
__device__ __forceinline__ bool aligned16_dev(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// ---- thread-block clusters: rank, barrier, distributed shared memory ---------------------
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Every thread of every CTA of the cluster arrives (its shared-memory writes released) and
// waits for all (acquiring theirs). Warp-convergent: all lanes execute it together.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// 32-bit word at shared-memory address `local` (this CTA's address space) of cluster CTA `rank`.
__device__ __forceinline__ uint32_t ld_dsmem_u32(uint32_t local, uint32_t rank) {
  uint32_t remote, v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(remote));
  return v;
}

// Word `rel` of probe p's mirror, computed from its hash table: 32 presence bits (slots
// 32 * rel ..) or eight 4-bit payload codes (slots 8 * rel ..); slots past the table are 0.
__device__ __forceinline__ uint32_t mirror_word(const StarPlan& P, int p, int rel) {
  const int slots = P.p_slots[p];
  const int* ht = P.p_ht[p];
  uint32_t w = 0;
  if (P.mir_kind[p] == kMirBits) {
    const int s0 = rel * 32;
    if (P.p_layout[p] == MB_HT_KEY) {
      if (s0 + 32 <= slots && aligned16_dev(ht)) {
        const int4* src = reinterpret_cast<const int4*>(ht + s0);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int4 q = __ldg(src + j);
          w |= ((q.x != 0 ? 1u : 0u) << (4 * j)) | ((q.y != 0 ? 1u : 0u) << (4 * j + 1)) |
               ((q.z != 0 ? 1u : 0u) << (4 * j + 2)) | ((q.w != 0 ? 1u : 0u) << (4 * j + 3));
        }
      } else {
        for (int j = 0; j < 32 && s0 + j < slots; ++j) w |= (__ldg(ht + s0 + j) != 0 ? 1u : 0u) << j;
      }
    } else {
      const unsigned long long* t8 = reinterpret_cast<const unsigned long long*>(ht);
      if (s0 + 32 <= slots && aligned16_dev(ht)) {
        const ulonglong2* src = reinterpret_cast<const ulonglong2*>(t8 + s0);
#pragma unroll 4
        for (int j = 0; j < 16; ++j) {
          const ulonglong2 q = __ldg(src + j);
          w |= ((q.x != 0ull ? 1u : 0u) << (2 * j)) | ((q.y != 0ull ? 1u : 0u) << (2 * j + 1));
        }
      } else {
        for (int j = 0; j < 32 && s0 + j < slots; ++j) w |= (__ldg(t8 + s0 + j) != 0ull ? 1u : 0u) << j;
      }
    }
    return w;
  }
  // payload codes: 0 absent, 1..14 payload - min + 1, 15 present with another payload
  const int s0 = rel * 8;
  const unsigned long long* t8 = reinterpret_cast<const unsigned long long*>(ht);
  const bool hi = P.p_layout[p] == MB_HT_KEY_VAL;
  const unsigned mn = static_cast<unsigned>(P.mir_min[p]);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (s0 + j >= slots) break;
    const unsigned long long v = __ldg(t8 + s0 + j);
    if (v == 0ull) continue;
    const unsigned pay = hi ? static_cast<unsigned>(v >> 32) : static_cast<unsigned>(v);
    const unsigned d = pay - mn;
    const unsigned code = d <= 13u ? d + 1u : kNibbleEscape;
    w |= code << (4 * j);
  }
  return w;
}

// This CTA's share of the cluster's mirror space (words rank << mir_shift ..), written by
// `nthreads` threads numbered t.
__device__ __forceinline__ void build_mirror_share(const StarPlan& P, uint32_t* share, int t, int nthreads) {
  const int words = 1 << P.mir_shift;
  const int w0 = static_cast<int>(cluster_rank()) << P.mir_shift;
  for (int i = t; i < words; i += nthreads) {
    const int gw = w0 + i;
    uint32_t word = 0;
    for (int p = 0; p < P.np; ++p) {
      if (P.mir_kind[p] == kMirNone) continue;
      const int rel = gw - P.mir_base[p];
      if (rel >= 0 && rel < P.mir_words[p]) {
        word = mirror_word(P, p, rel);
        break;
      }
    }
    share[i] = word;
  }
}

// Column pointer for row `r` of this call (direct or through the segment cache).
__device__ __forceinline__ const int* row_ptr(const StarPlan& P, int c, long long r) {
  if (P.gpu_cache == nullptr) return P.col[c] + r;
  const long long vseg = r >> P.seg_shift;
  const int seg = P.seg_group ? static_cast<int>(P.seg_group[vseg])
                              : static_cast<int>((P.start_offset + r) >> P.seg_shift);
  const long long slot = P.col[c][seg];
  return P.gpu_cache + (slot << P.seg_shift) + (r & ((1ll << P.seg_shift) - 1));
}

// Loaders hand the sparse phase a column's values for the rows it holds: load(slot, c, v)
// reads staged column c. `slot` names the column's role — sparse position q for a probe
// key, kAggSlot + a for aggregate column a — and is a compile-time constant after
// unrolling; only RegLoader uses it.
constexpr int kAggSlot = MB_MAX_PROBES;
constexpr int kLoadSlots = MB_MAX_PROBES + 2;

// Survivors gathered from a staged tile through a warp's row list.
template <int TILE, int R>
struct GatherLoader {
  static constexpr int ITEMS = R;
  const int* wstage;
  int r[R];
  __device__ __forceinline__ void load(int, int c, int (&v)[R]) const {
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = wstage[c * TILE + r[i]];
  }
};

// Survivors whose columns were copied into registers (the stage they came from already
// returned to the producer).
template <int R>
struct RegLoader {
  static constexpr int ITEMS = R;
  int val[kLoadSlots][R];
  __device__ __forceinline__ void load(int slot, int, int (&v)[R]) const {
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = val[slot][i];
  }
};

// One remainder row read straight from global memory.
struct RowLoader {
  static constexpr int ITEMS = 1;
  const StarPlan* P;
  long long r;
  __device__ __forceinline__ void load(int, int c, int (&v)[1]) const { v[0] = __ldg(row_ptr(*P, c, r)); }
};

// Probe index of sparse position q. The tiled path visits its sparse probes in the
// planned order P.sp_ord (the first probe that can drop rows first, ahead of probes the
// dense phase already settled and that are read only for their payloads); rows read
// without a dense phase (the remainder) visit them in chain order from p0.
template <bool ORD>
__device__ __forceinline__ int sparse_probe(const StarPlan& P, int p0, int q) {
  return ORD ? P.sp_ord[q] : p0 + q;
}

// Key columns of group h from the payloads of the sparse table probes (gv[q] = sparse
// position q). Bitmap-decided probes have payload 0 and the caller zeroed the result, so
// they are not written.
template <int NSC, int ITEMS, bool ORD>
__device__ __forceinline__ void write_keys(const StarPlan& P, int h, const int (&gv)[MB_MAX_PROBES][ITEMS], int i,
                                           int p0, int ns) {
  int* res = static_cast<int*>(P.res);
  const int stride = P.res_layout == MB_RES_ENGINE6 ? 6 : 4;
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q) {
    if (q >= (NSC >= 0 ? NSC : ns)) break;
    const int rs = P.p_res_slot[sparse_probe<ORD>(P, p0, q)];
    if (rs >= 0) res[stride * h + rs] = gv[q][i];
  }
}

__device__ __forceinline__ unsigned long long* group_sum_ptr(const StarPlan& P, int h) {
  if (P.res_layout == MB_RES_ENGINE6)
    return reinterpret_cast<unsigned long long*>(static_cast<int*>(P.res) + 6 * h + 4);
  if (P.res_layout == MB_RES_CRYSTAL4)
    return reinterpret_cast<unsigned long long*>(static_cast<int*>(P.res) + 4 * h + 2);
  return static_cast<unsigned long long*>(P.res) + h;
}

struct Accum {
  unsigned long long acc = 0, cnt = 0;
  bool bad_probe = false, bad_group = false;
};

// Aggregate the rows still selected in `sel` into the scalar or the groups. gv[q] is the
// payload of table probe p0 + q; `bias` already holds the group terms of every probe
// before p0 (bitmap-decided probes, payload 0).
template <int NSC, int ITEMS, bool ORD, class L>
__device__ __forceinline__ void aggregate_rows(const StarPlan& P, const L& ld, uint32_t sel,
                                               const int (&gv)[MB_MAX_PROBES][ITEMS], int p0, int ns,
                                               unsigned bias, Accum& A, unsigned long long* s_sum,
                                               uint32_t* s_touch) {
  int a0[ITEMS], a1[ITEMS];
  ld.load(kAggSlot, P.a_col[0], a0);
  if (P.agg_op == MB_AGG_SUB || P.agg_op == MB_AGG_MUL) ld.load(kAggSlot + 1, P.a_col[1], a1);
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
      A.acc += w;
      continue;
    }
    unsigned hh = bias;
#pragma unroll
    for (int q = 0; q < MB_MAX_PROBES; ++q) {
      if (q >= (NSC >= 0 ? NSC : ns)) break;
      const int p = sparse_probe<ORD>(P, p0, q);
      hh += (static_cast<unsigned>(gv[q][i]) - static_cast<unsigned>(P.p_min[p])) * static_cast<unsigned>(P.p_mul[p]);
    }
    int h = static_cast<int>(hh);
    if (static_cast<unsigned>(h) >= static_cast<unsigned>(P.total_val)) h = slow_mod(h, P.total_val);
    if (h < 0) {
      A.bad_group = true;
      continue;
    }
    if (P.gmode == kGroupSmem) {
      atomicAdd(&s_sum[h], w);
      const uint32_t bit = 1u << (h & 31);
      if (!(s_touch[h >> 5] & bit)) {
        if (!(atomicOr(&s_touch[h >> 5], bit) & bit) && P.res_layout != MB_RES_DENSE)
          write_keys<NSC, ITEMS, ORD>(P, h, gv, i, p0, ns);
      }
    } else {
      if (P.res_layout != MB_RES_DENSE) write_keys<NSC, ITEMS, ORD>(P, h, gv, i, p0, ns);
      atomicAdd(group_sum_ptr(P, h), w);
    }
  }
}

// One round of table probes: probes p0 + q for q in [qlo, qhi) (and q < nsp) for the rows
// in `sel`. Every probe's loads go out before any is checked; presence is then combined
// probe by probe in order, so selection, payloads (gv[q]) and status bits equal the
// sequential chain.
template <int ITEMS, bool ORD, class L>
__device__ __forceinline__ void probe_round(const StarPlan& P, const L& ld, uint32_t& sel, int p0, int nsp, int qlo,
                                            int qhi, int (&gv)[MB_MAX_PROBES][ITEMS], Accum& A,
                                            const unsigned char* smem) {
  int v[ITEMS];
  unsigned long long sv[MB_MAX_PROBES][ITEMS];
  uint32_t range_bad[MB_MAX_PROBES], absent[MB_MAX_PROBES];
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q) {
    range_bad[q] = 0;
    absent[q] = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) sv[q][i] = 0;
  }
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q) {
    if (q >= nsp) break;
    if (q < qlo || q >= qhi) continue;
    const int p = sparse_probe<ORD>(P, p0, q);
    ld.load(q, P.p_col[p], v);
    const int slots = P.p_slots[p], kmin = P.p_kmin[p], layout = P.p_layout[p];
    const int* ht = P.p_ht[p];
    const uint32_t* bm = P.p_bm_off[p] >= 0 ? reinterpret_cast<const uint32_t*>(smem + P.p_bm_off[p]) : nullptr;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (sel & (1u << i)) {
        const int h = pht_slot(v[i], slots, kmin);
        if (h < 0)
          range_bad[q] |= 1u << i;
        else if (bm != nullptr && !((bm[h >> 5] >> (h & 31)) & 1u))
          absent[q] |= 1u << i;
        else if (layout == MB_HT_KEY)
          sv[q][i] = bm != nullptr ? 1ull : static_cast<unsigned long long>(static_cast<unsigned>(__ldg(ht + h)));
        else
          sv[q][i] = ldg_u64(ht + 2 * h);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q) {
    if (q >= nsp) break;
    if (q < qlo || q >= qhi) continue;
    const int layout = P.p_layout[sparse_probe<ORD>(P, p0, q)];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (!(sel & (1u << i))) continue;
      if (range_bad[q] & (1u << i)) {
        A.bad_probe = true;
        sel &= ~(1u << i);
      } else if ((absent[q] & (1u << i)) || sv[q][i] == 0) {
        sel &= ~(1u << i);
      } else {
        gv[q][i] = layout == MB_HT_KEY_VAL   ? static_cast<int>(sv[q][i] >> 32)
                   : layout == MB_HT_VAL_OFF ? static_cast<int>(static_cast<unsigned>(sv[q][i]))
                                             : 0;
      }
    }
  }
}

// Table probes p0 .. p0+ns-1 and the aggregate for the rows a loader exposes, in two
// rounds: the first table probe alone, then the others together for the rows it kept
// (the first probe removes most rows, so later tables see a fraction of the loads, at
// the price of one more L2 round trip). Per lane: usable from divergent code.
template <int NSC, bool ORD, class L>
__device__ __forceinline__ void sparse_rows(const StarPlan& P, const L& ld, uint32_t sel, int p0, int ns,
                                            unsigned bias, Accum& A, unsigned long long* s_sum, uint32_t* s_touch,
                                            const unsigned char* smem) {
  constexpr int ITEMS = L::ITEMS;
  if (sel == 0) return;
  int gv[MB_MAX_PROBES][ITEMS];
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q)
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) gv[q][i] = 0;
  const int nsp = NSC >= 0 ? NSC : ns;
  probe_round<ITEMS, ORD>(P, ld, sel, p0, nsp, 0, 1, gv, A, smem);
  if (sel == 0) return;
  probe_round<ITEMS, ORD>(P, ld, sel, p0, nsp, 1, MB_MAX_PROBES, gv, A, smem);
  if (P.count_after < 0) A.cnt += __popc(sel);
  if (sel == 0) return;
  aggregate_rows<NSC, ITEMS, ORD>(P, ld, sel, gv, p0, ns, bias, A, s_sum, s_touch);
}

// Lane of the (k+1)-th set bit of `mask` (k < popc(mask)).
__device__ __forceinline__ int nth_set_lane(uint32_t mask, int k) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (__popc(mask & ((2u << (lo + step - 1)) - 1u)) <= k) lo += step;
  return lo;
}

// sparse_rows for a warp's batch of R survivors a lane, with the warp converged (every
// lane calls it): after the first probe the rows it kept — about one in five — are packed
// across the warp, one a lane (row offset and first payload moved by shuffles), so the
// second round and the aggregate run once over full lanes instead of R times over mostly
// empty ones.
template <int NSC, int TILE, int R>
__device__ __forceinline__ void sparse_rows_packed(const StarPlan& P, const GatherLoader<TILE, R>& ld, uint32_t sel,
                                                   int p0, int ns, unsigned bias, Accum& A,
                                                   unsigned long long* s_sum, uint32_t* s_touch,
                                                   const unsigned char* smem) {
  const int nsp = NSC >= 0 ? NSC : ns;
  if (nsp < 2) {  // no second round to pack for
    sparse_rows<NSC, true>(P, ld, sel, p0, ns, bias, A, s_sum, s_touch, smem);
    return;
  }
  const int lane = threadIdx.x & 31;
  int gv0[MB_MAX_PROBES][R];
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q)
#pragma unroll
    for (int i = 0; i < R; ++i) gv0[q][i] = 0;
  probe_round<R, true>(P, ld, sel, p0, nsp, 0, 1, gv0, A, smem);
  uint32_t b[R];
  int c[R], total = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    b[i] = __ballot_sync(kFull, (sel >> i) & 1u);
    c[i] = __popc(b[i]);
    total += c[i];
  }
  // survivors in item-major order: every lane's item 0, then every lane's item 1, ...
  for (int base = 0; base < total; base += 32) {
    int rem = base + lane, row = 0, g = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const bool mine = rem >= 0 && rem < c[i];
      const int src = mine ? nth_set_lane(b[i], rem) : lane;
      const int xr = __shfl_sync(kFull, ld.r[i], src);
      const int xg = __shfl_sync(kFull, gv0[0][i], src);
      if (mine) {
        row = xr;
        g = xg;
      }
      rem -= c[i];
    }
    GatherLoader<TILE, 1> l1;
    l1.wstage = ld.wstage;
    l1.r[0] = row;
    uint32_t s1 = base + lane < total ? 1u : 0u;
    int gv[MB_MAX_PROBES][1];
#pragma unroll
    for (int q = 0; q < MB_MAX_PROBES; ++q) gv[q][0] = 0;
    gv[0][0] = g;
    probe_round<1, true>(P, l1, s1, p0, nsp, 1, MB_MAX_PROBES, gv, A, smem);
    if (P.count_after < 0) A.cnt += s1;
    if (s1) aggregate_rows<NSC, 1, true>(P, l1, s1, gv, p0, ns, bias, A, s_sum, s_touch);
  }
}

// The columns the sparse phase reads for a batch (every sparse probe key, the aggregate
// operands), copied from the stage into registers.
template <int NSC, int TILE, int R>
__device__ __forceinline__ void copy_to_regs(const StarPlan& P, const GatherLoader<TILE, R>& gl, int p0, int ns,
                                             RegLoader<R>& rl) {
  const int nsp = NSC >= 0 ? NSC : ns;
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q) {
    if (q >= nsp) break;
    gl.load(q, P.p_col[sparse_probe<true>(P, p0, q)], rl.val[q]);
  }
  gl.load(kAggSlot, P.a_col[0], rl.val[kAggSlot]);
  if (P.agg_op == MB_AGG_SUB || P.agg_op == MB_AGG_MUL) gl.load(kAggSlot + 1, P.a_col[1], rl.val[kAggSlot + 1]);
}

// sparse_rows for a warp's last batch of a tile, returning the stage early: the batch's
// columns go to registers, `release()` hands the stage back, and both probe rounds run
// from registers. Warp-converged.
template <int NSC, int TILE, int R, class Release>
__device__ __forceinline__ void sparse_rows_regs(const StarPlan& P, const GatherLoader<TILE, R>& gl, uint32_t sel,
                                                 int p0, int ns, unsigned bias, Accum& A, unsigned long long* s_sum,
                                                 uint32_t* s_touch, const unsigned char* smem, Release release) {
  RegLoader<R> rl;
  copy_to_regs<NSC>(P, gl, p0, ns, rl);
  release();
  sparse_rows<NSC, true>(P, rl, sel, p0, ns, bias, A, s_sum, s_touch, smem);
}

// sparse_rows_packed for a warp's last batch of a tile, returning the stage early: the
// survivors' columns that the sparse phase reads (every sparse probe key and the
// aggregate operands) are copied into registers, `release()` hands the stage back to
// the producer, and the two probe rounds — with their L2 round trips — run from
// registers while the next tile lands. After the first probe each kept row is written,
// with its payload and its other columns, to its packed position (item-major: every
// lane's item 0 first) in the warp's buffer `xfer` (the survivor list, read already:
// 32 rows of kXferWords ints), and each lane reads one packed row back — a scatter, with
// no search for source lanes. Warp-converged: every lane calls it.
template <int NSC, int TILE, int R, class Release>
__device__ __forceinline__ void sparse_rows_packed_regs(const StarPlan& P, const GatherLoader<TILE, R>& gl,
                                                        uint32_t sel, int p0, int ns, unsigned bias, Accum& A,
                                                        unsigned long long* s_sum, uint32_t* s_touch,
                                                        const unsigned char* smem, int* xfer, Release release) {
  static_assert(kXferWords >= kLoadSlots, "a packed row holds the payload and every column slot");
  const int nsp = NSC >= 0 ? NSC : ns;
  const bool two_ops = P.agg_op == MB_AGG_SUB || P.agg_op == MB_AGG_MUL;
  RegLoader<R> rl;
  copy_to_regs<NSC>(P, gl, p0, ns, rl);
  release();
  if (nsp < 2) {
    sparse_rows<NSC, true>(P, rl, sel, p0, ns, bias, A, s_sum, s_touch, smem);
    return;
  }
  const int lane = threadIdx.x & 31;
  int gv0[MB_MAX_PROBES][R];
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q)
#pragma unroll
    for (int i = 0; i < R; ++i) gv0[q][i] = 0;
  probe_round<R, true>(P, rl, sel, p0, nsp, 0, 1, gv0, A, smem);
  uint32_t b[R];
  int c[R], total = 0;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    b[i] = __ballot_sync(kFull, (sel >> i) & 1u);
    c[i] = __popc(b[i]);
    total += c[i];
  }
  const uint32_t below = (1u << lane) - 1u;
  // slot j of a packed row: 0 the first probe's payload, 1..nsp-1 the later probe keys,
  // kAggSlot.. the aggregate operands
  auto used = [&](int j) { return !(j < MB_MAX_PROBES && j >= nsp) && !(j == kAggSlot + 1 && !two_ops); };
  for (int base = 0; base < total; base += 32) {
    int first = -base;  // packed position of this group's first row of item i
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int pos = first + __popc(b[i] & below);
      if (((sel >> i) & 1u) && pos >= 0 && pos < 32) {
        int* dst = xfer + pos * kXferWords;
        dst[0] = gv0[0][i];
#pragma unroll
        for (int j = 1; j < kLoadSlots; ++j)
          if (used(j)) dst[j] = rl.val[j][i];
      }
      first += c[i];
    }
    __syncwarp();
    RegLoader<1> r1;
    const int* src = xfer + lane * kXferWords;
    int gv[MB_MAX_PROBES][1];
#pragma unroll
    for (int q = 0; q < MB_MAX_PROBES; ++q) gv[q][0] = 0;
    gv[0][0] = src[0];
#pragma unroll
    for (int j = 1; j < kLoadSlots; ++j) r1.val[j][0] = used(j) ? src[j] : 0;
    __syncwarp();  // every read done before the next group's writes or the list's next use
    uint32_t s1 = base + lane < total ? 1u : 0u;
    probe_round<1, true>(P, r1, s1, p0, nsp, 1, MB_MAX_PROBES, gv, A, smem);
    if (P.count_after < 0) A.cnt += s1;
    if (s1) aggregate_rows<NSC, 1, true>(P, r1, s1, gv, p0, ns, bias, A, s_sum, s_touch);
  }
}

// The sparse phase with cluster-resident mirrors: a probe with a mirror tests presence —
// and, with payload codes, reads the payload — in the cluster's distributed shared memory
// instead of L2; probes without one read their tables as in sparse_rows. Payloads a mirror
// does not hold (presence-bit mirrors of tables whose payload is read, escaped codes) are
// read from the table for the rows that survive every probe. Selection, payloads and
// status bits equal the sequential chain's.
template <int NSC, class L>
__device__ __forceinline__ void sparse_rows_mir(const StarPlan& P, const L& ld, uint32_t sel, int p0, int ns,
                                                unsigned bias, Accum& A, unsigned long long* s_sum, uint32_t* s_touch,
                                                const unsigned char* smem) {
  constexpr int ITEMS = L::ITEMS;
  if (sel == 0) return;
  int v[ITEMS];
  int gv[MB_MAX_PROBES][ITEMS];
  unsigned long long sv[MB_MAX_PROBES][ITEMS];
  uint32_t range_bad[MB_MAX_PROBES], absent[MB_MAX_PROBES], fetch[MB_MAX_PROBES];
#pragma unroll
  for (int p = 0; p < MB_MAX_PROBES; ++p) {
    range_bad[p] = 0;
    absent[p] = 0;
    fetch[p] = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      gv[p][i] = 0;
      sv[p][i] = 0;
    }
  }
  const uint32_t share = smem_addr(smem + P.smem_mirror_off);
  const int smask = (1 << P.mir_shift) - 1;
  const int nsp = NSC >= 0 ? NSC : ns;
#pragma unroll
  for (int round = 0; round < 2; ++round) {
    const int qlo = round == 0 ? 0 : 1, qhi = round == 0 ? 1 : MB_MAX_PROBES;
#pragma unroll
    for (int q = 0; q < MB_MAX_PROBES; ++q) {
      if (q >= nsp) break;
      if (q < qlo || q >= qhi) continue;
      const int p = p0 + q;
      ld.load(q, P.p_col[p], v);
      const int slots = P.p_slots[p], kmin = P.p_kmin[p], layout = P.p_layout[p], kind = P.mir_kind[p];
      const int base = P.mir_base[p];
      const int* ht = P.p_ht[p];
      const uint32_t* bm = P.p_bm_off[p] >= 0 ? reinterpret_cast<const uint32_t*>(smem + P.p_bm_off[p]) : nullptr;
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        if (!(sel & (1u << i))) continue;
        const int h = pht_slot(v[i], slots, kmin);
        if (h < 0) {
          range_bad[q] |= 1u << i;
        } else if (bm != nullptr && !((bm[h >> 5] >> (h & 31)) & 1u)) {
          absent[q] |= 1u << i;
        } else if (kind == kMirBits) {
          const int gw = base + (h >> 5);
          sv[q][i] = (ld_dsmem_u32(share + 4u * static_cast<uint32_t>(gw & smask), static_cast<uint32_t>(gw) >> P.mir_shift) >>
                      (h & 31)) & 1u;
        } else if (kind == kMirNibble) {
          const int gw = base + (h >> 3);
          sv[q][i] = (ld_dsmem_u32(share + 4u * static_cast<uint32_t>(gw & smask), static_cast<uint32_t>(gw) >> P.mir_shift) >>
                      (4 * (h & 7))) & 15u;
        } else if (layout == MB_HT_KEY) {
          sv[q][i] = bm != nullptr ? 1ull : static_cast<unsigned long long>(static_cast<unsigned>(__ldg(ht + h)));
        } else {
          sv[q][i] = ldg_u64(ht + 2 * h);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < MB_MAX_PROBES; ++q) {
      if (q >= nsp) break;
      if (q < qlo || q >= qhi) continue;
      const int p = p0 + q;
      const int layout = P.p_layout[p], kind = P.mir_kind[p];
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) {
        if (!(sel & (1u << i))) continue;
        if (range_bad[q] & (1u << i)) {
          A.bad_probe = true;
          sel &= ~(1u << i);
        } else if ((absent[q] & (1u << i)) || sv[q][i] == 0) {
          sel &= ~(1u << i);
        } else if (kind == kMirBits) {
          if (P.mir_payload[p]) fetch[q] |= 1u << i;
        } else if (kind == kMirNibble) {
          if (sv[q][i] == kNibbleEscape)
            fetch[q] |= 1u << i;
          else
            gv[q][i] = static_cast<int>(static_cast<unsigned>(P.mir_min[p]) + static_cast<unsigned>(sv[q][i]) - 1u);
        } else {
          gv[q][i] = layout == MB_HT_KEY_VAL   ? static_cast<int>(sv[q][i] >> 32)
                     : layout == MB_HT_VAL_OFF ? static_cast<int>(static_cast<unsigned>(sv[q][i]))
                                               : 0;
        }
      }
    }
    if (sel == 0) return;  // per lane; nothing warp-wide follows
  }
  // payloads the mirrors do not hold, for the rows that passed every probe
#pragma unroll
  for (int q = 0; q < MB_MAX_PROBES; ++q) {
    if (q >= nsp) break;
    if (!(fetch[q] & sel)) continue;
    const int p = p0 + q;
    ld.load(q, P.p_col[p], v);
    const int* ht = P.p_ht[p];
    const bool hi = P.p_layout[p] == MB_HT_KEY_VAL;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      if (!(fetch[q] & sel & (1u << i))) continue;
      const unsigned long long raw = ldg_u64(ht + 2 * pht_slot(v[i], P.p_slots[p], P.p_kmin[p]));
      gv[q][i] = hi ? static_cast<int>(raw >> 32) : static_cast<int>(static_cast<unsigned>(raw));
    }
  }
  if (P.count_after < 0) A.cnt += __popc(sel);
  aggregate_rows<NSC, ITEMS, false>(P, ld, sel, gv, p0, ns, bias, A, s_sum, s_touch);
}

// Dense phase over a warp's slice of a staged tile: lane l owns rows (j*32 + l)*4 + e,
// read with 128-bit shared loads; applies every filter and the leading probes whose
// presence bitmap is staged. Returns the selection (bit j*4 + e).
template <int NFC, int NDC, int ITEMS, int TILE>
__device__ __forceinline__ uint32_t dense_phase(const StarPlan& P, const int* wstage, const unsigned char* smem,
                                                Accum& A) {
  const int lane = threadIdx.x & 31;
  uint32_t sel = ITEMS == 32 ? kFull : ((1u << ITEMS) - 1u);
  int v[ITEMS];
  auto load = [&](int c) {
#pragma unroll
    for (int j = 0; j < ITEMS / 4; ++j) {
      const int4 q = lds128(wstage + c * TILE + (j * 32 + lane) * 4);
      v[4 * j + 0] = q.x;
      v[4 * j + 1] = q.y;
      v[4 * j + 2] = q.z;
      v[4 * j + 3] = q.w;
    }
  };
  const int nf = NFC >= 0 ? NFC : P.nf;
#pragma unroll
  for (int f = 0; f < MB_MAX_FILTERS; ++f) {
    if (f >= nf) break;
    if (P.count_after == f) A.cnt += __popc(sel);
    if (f > 0 && !__any_sync(kFull, sel != 0)) continue;
    load(P.f_col[f]);
    const int mode = P.f_mode[f], c1 = P.f_c1[f], c2 = P.f_c2[f];
    if (mode == MB_FILTER_BETWEEN) {
      // c1 <= x <= c2  <=>  (unsigned)(x - c1) <= (unsigned)(c2 - c1), for c1 <= c2
      const unsigned span = static_cast<unsigned>(c2) - static_cast<unsigned>(c1);
      if (c2 < c1) sel = 0;
#pragma unroll
      for (int i = 0; i < ITEMS; ++i)
        if (static_cast<unsigned>(v[i]) - static_cast<unsigned>(c1) > span) sel &= ~(1u << i);
    } else {
#pragma unroll
      for (int i = 0; i < ITEMS; ++i)
        if (!pass_filter(v[i], mode, c1, c2)) sel &= ~(1u << i);
    }
  }
  if (P.count_after >= nf) A.cnt += __popc(sel);
  const int nd = NDC >= 0 ? NDC : P.n_dense;
#pragma unroll
  for (int p = 0; p < MB_MAX_PROBES; ++p) {
    if (p >= nd) break;
    if ((p > 0 || nf > 0) && !__any_sync(kFull, sel != 0)) break;
    load(P.p_col[p]);
    const uint32_t* bm = reinterpret_cast<const uint32_t*>(smem + P.p_bm_off[p]);
    const int slots = P.p_slots[p], kmin = P.p_kmin[p];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const int h = pht_slot(v[i], slots, kmin);
      if (h < 0) {
        if (sel & (1u << i)) A.bad_probe = true;
        sel &= ~(1u << i);
      } else if (!((bm[h >> 5] >> (h & 31)) & 1u)) {
        sel &= ~(1u << i);
      }
    }
  }
  return sel;
}

// Warp prefix sum of the selection counts; writes survivor row offsets to `list`.
__device__ __forceinline__ int compact(uint32_t sel, uint16_t* list) {
  const int lane = threadIdx.x & 31;
  const int c = __popc(sel);
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  int pos = incl - c;
  __syncwarp();  // the previous tile's readers of `list` are done
  while (sel) {
    const int i = __ffs(sel) - 1;
    sel &= sel - 1;
    list[pos++] = static_cast<uint16_t>(((i >> 2) * 32 + lane) * 4 + (i & 3));
  }
  __syncwarp();
  return total;
}

// Generic per-row path (remainder rows): every filter and probe with run-time counts.
template <class L>
__device__ __forceinline__ void tail_row(const StarPlan& P, const L& ld, Accum& A, unsigned long long* s_sum,
                                         uint32_t* s_touch, const unsigned char* smem) {
  uint32_t sel = 1u;
  int v[1];
  for (int f = 0; f < P.nf; ++f) {
    if (P.count_after == f) A.cnt += sel;
    if (!sel) continue;
    ld.load(-1, P.f_col[f], v);
    if (!pass_filter(v[0], P.f_mode[f], P.f_c1[f], P.f_c2[f])) sel = 0;
  }
  if (P.count_after >= P.nf) A.cnt += sel;
  // bitmap-decided probes run here as table probes (sparse_rows consults a staged bitmap)
  sparse_rows<-1, false>(P, ld, sel, 0, P.np, static_cast<unsigned>(P.group_bias), A, s_sum, s_touch, smem);
}

// CTAs per SM the register budget must allow for a variant of NCW consumer warps: the
// small-CTA shapes run two (8 warps) or four (4 warps) CTAs an SM where their stages fit,
// and a register or two more per thread would cost a whole CTA (each scheduler's 16 K
// registers are split among its warps).
constexpr int star_min_ctas(int ncw) { return ncw <= 4 ? 4 : ncw <= 8 ? 2 : 1; }

template <int NCW, int ITEMS, int NFC, int NDC, int NSC, bool MIR = false, bool PACK = false, bool REL = false>
__global__ void __launch_bounds__((NCW + 1) * 32, star_min_ctas(NCW)) star_kernel(const __grid_constant__ StarPlan P) {
  constexpr int WROWS = 32 * ITEMS;
  constexpr int NSL = tile_slices(NCW);
  constexpr int TILE = NSL * WROWS;
  constexpr int NWARPS = NCW + 1;
  constexpr int R = ITEMS / 4 < 2 ? 2 : ITEMS / 4;  // survivors per lane per sparse round
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long s_red[2 * NWARPS];

  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + 2 * kMaxStages;
  unsigned long long* s_sum = reinterpret_cast<unsigned long long*>(smem + P.smem_groups_off);
  uint32_t* s_touch = reinterpret_cast<uint32_t*>(smem + P.smem_groups_off + 8 * P.total_val);
  int* stage_base = reinterpret_cast<int*>(smem + P.smem_stage_off);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = P.stages;

  // ---- set-up: group accumulators, staged presence bitmaps, barriers ----------
  if (P.gmode == kGroupSmem) {
    for (int g = tid; g < P.total_val; g += NWARPS * 32) s_sum[g] = 0;
    for (int w = tid; w < (P.total_val + 31) / 32; w += NWARPS * 32) s_touch[w] = 0;
  }
  for (int p = 0; p < P.np; ++p) {
    if (P.p_bm_off[p] < 0) continue;
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem + P.p_bm_off[p]);
    const int words = P.p_bm_words[p];
    if (P.p_presence[p] != nullptr) {
      for (int w = tid; w < words; w += NWARPS * 32) bm[w] = __ldg(P.p_presence[p] + w);
    } else if (P.p_layout[p] != MB_HT_KEY) {
      // derive presence from a table with 8-byte slots: slot s is present when nonzero
      const int slots = P.p_slots[p];
      const unsigned long long* ht = reinterpret_cast<const unsigned long long*>(P.p_ht[p]);
      const bool vec = aligned16_dev(ht);
      for (int w = tid; w < words; w += NWARPS * 32) {
        uint32_t word = 0;
        if (vec && (w + 1) * 32 <= slots) {
          // four 16-byte loads (8 slots) in flight at a time: few registers, so the set-up
          // does not raise the kernel's register count
          const ulonglong2* src = reinterpret_cast<const ulonglong2*>(ht + w * 32);
#pragma unroll 1
          for (int j0 = 0; j0 < 16; j0 += 4) {
            ulonglong2 q[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) q[j] = __ldg(src + j0 + j);
#pragma unroll
            for (int j = 0; j < 4; ++j)
              word |= ((q[j].x != 0ull ? 1u : 0u) << (2 * (j0 + j))) | ((q[j].y != 0ull ? 1u : 0u) << (2 * (j0 + j) + 1));
          }
        } else {
          for (int j = 0; j < 32 && w * 32 + j < slots; ++j) word |= (__ldg(ht + w * 32 + j) != 0ull ? 1u : 0u) << j;
        }
        bm[w] = word;
      }
    } else {
      // derive presence from an MB_HT_KEY table: each thread folds 32 slots into a word
      // with its eight 16-byte loads in flight together
      const int slots = P.p_slots[p];
      const int* ht = P.p_ht[p];
      const bool vec = aligned16_dev(ht);
      for (int w = tid; w < words; w += NWARPS * 32) {
        uint32_t word = 0;
        if (vec && (w + 1) * 32 <= slots) {
          int4 q[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) q[j] = __ldg(reinterpret_cast<const int4*>(ht + w * 32) + j);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            word |= ((q[j].x != 0 ? 1u : 0u) << (4 * j)) | ((q[j].y != 0 ? 1u : 0u) << (4 * j + 1)) |
                    ((q[j].z != 0 ? 1u : 0u) << (4 * j + 2)) | ((q[j].w != 0 ? 1u : 0u) << (4 * j + 3));
        } else {
          for (int j = 0; j < 32 && w * 32 + j < slots; ++j) word |= (__ldg(ht + w * 32 + j) != 0 ? 1u : 0u) << j;
        }
        bm[w] = word;
      }
    }
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&full[S + s], 1);
      mbar_init(&empty[s], NSL);
    }
    mbar_fence_init();
  }
  __syncthreads();

  const long long G = gridDim.x;
  const long long b = blockIdx.x;
  const long long my_tiles = P.nfull > b ? (P.nfull - 1 - b) / G + 1 : 0;
  const uint32_t stage_words = static_cast<uint32_t>(P.ncols) * TILE;
  Accum A;
  bool failed = false;

  if (warp == 0) {
    // ---- producer: one lane streams tiles into the stage ring ----------------------
    const uint64_t policy = l2_policy_evict_first();
    long long k = 0;
    int s = 0;
    uint32_t phase = 0;  // use count of stage s, mod 2
    // tile kk goes to stage ss = kk % S and lands on full barrier kk % 2S = ss + S * (use
    // count of the stage mod 2)
    auto issue = [&](long long kk, int ss, uint32_t use) {
      const long long r0 = (b + kk * G) * static_cast<long long>(TILE);
      int* dst = stage_base + ss * stage_words;
      fence_proxy_async_smem();
      uint64_t* fb = &full[ss + S * static_cast<int>(use)];
      mbar_arrive_expect_tx(fb, stage_words * 4u);
      if (P.gpu_cache == nullptr) {
        for (int c = 0; c < P.ncols; ++c) bulk_g2s(dst + c * TILE, P.col[c] + r0, TILE * 4, fb, policy);
      } else {
        const long long vseg = r0 >> P.seg_shift;
        const int seg = P.seg_group ? static_cast<int>(P.seg_group[vseg])
                                    : static_cast<int>((P.start_offset + r0) >> P.seg_shift);
        const long long in_seg = r0 & ((1ll << P.seg_shift) - 1);
        // every column's cache slot first (independent loads in flight together), then
        // the copies: a copy is an ordered asm statement, so a slot load placed between
        // two copies would wait for the previous load to return
        int slot[kMaxCols];
#pragma unroll
        for (int c = 0; c < kMaxCols; ++c)
          if (c < P.ncols) slot[c] = P.col[c][seg];
#pragma unroll
        for (int c = 0; c < kMaxCols; ++c)
          if (c < P.ncols)
            bulk_g2s(dst + c * TILE, P.gpu_cache + (static_cast<long long>(slot[c]) << P.seg_shift) + in_seg,
                     TILE * 4, fb, policy);
      }
    };
    if (MIR) {
      // fill the ring while the consumers build the mirrors, then join the cluster barrier
      if (lane == 0) {
        for (; k < my_tiles && k < S; ++k) {
          issue(k, s, phase);
          if (++s == S) {
            s = 0;
            phase ^= 1u;
          }
        }
      }
      __syncwarp();
      cluster_sync_all();
    }
    if (lane == 0) {
      for (; k < my_tiles; ++k) {
        if (k >= S && !mbar_wait_bounded(&empty[s], phase ^ 1u)) {
          failed = true;
          break;
        }
        issue(k, s, phase);
        if (++s == S) {
          s = 0;
          phase ^= 1u;
        }
      }
      // no copy may land after the CTA is gone: wait (bounded) for the last ones issued
      for (long long j = (k > S ? k - S : 0); j < k; ++j)
        if (!mbar_wait_bounded(&full[j % (2 * S)], static_cast<uint32_t>((j / (2 * S)) & 1))) failed = true;
    }
  } else {
    // ---- consumers ---------------------------------------------------------------------
    const int cw = warp - 1;
    constexpr int LIST_BYTES = star_list_bytes(ITEMS, PACK && REL);
    uint16_t* list = reinterpret_cast<uint16_t*>(smem + P.smem_list_off + cw * LIST_BYTES);
    const int nd = P.sparse_p0;  // the sparse phase starts at probe sparse_p0 <= n_dense
    const int ns = NSC >= 0 ? NSC : P.np - P.sparse_p0;
    const unsigned sparse_bias = static_cast<unsigned>(P.group_bias) + P.dense_bias;
    if (MIR) {
      // this CTA's share of the mirrors, visible cluster-wide after the barrier
      build_mirror_share(P, reinterpret_cast<uint32_t*>(smem + P.smem_mirror_off), tid - 32, NCW * 32);
      __syncwarp();
      cluster_sync_all();
    }
    // Slice j of this CTA's sequence is slice j % NSL of tile j / NSL; warp cw takes
    // slices cw, cw + NCW, ... (with NCW == NSL: slice cw of every tile). Tile k lands on
    // full barrier k % 2S, two per stage: a warp that skipped tiles can wait for tile k
    // while tile k - S, on the same stage, is still landing, and a barrier shared by the
    // two would show tile k - S's phase. The previous use of barrier k % 2S is tile
    // k - 2S, which was consumed — so landed — before tile k - S was issued, and tile
    // k - S was issued before the tile of this warp's previous slice (at most two tiles
    // back, NCW <= 2 NSL; S >= 2), so the parity wait below is exact.
    static_assert(NCW <= 2 * NSL, "a warp's consecutive slices must be less than two tiles apart");
    long long k = 0;                   // tile of the current slice
    int sl = cw, s = 0, fb = 0;        // slice in the tile, stage k % S, full barrier k % 2S
    uint32_t par = 0;                  // parity of tile k's phase on barrier fb
    auto next_tile = [&]() {
      ++k;
      if (++s == S) s = 0;
      if (++fb == 2 * S) {
        fb = 0;
        par ^= 1u;
      }
    };
    while (sl >= NSL) {
      sl -= NSL;
      next_tile();
    }
    for (; k < my_tiles;) {
      const bool ok = mbar_wait_bounded(&full[fb], par);
      if (!__all_sync(kFull, ok)) {
        failed = true;
        break;
      }
      const int* wstage = stage_base + s * stage_words + sl * WROWS;
      const uint32_t sel = dense_phase<NFC, NDC, ITEMS, TILE>(P, wstage, smem, A);
      const int total = compact(sel, list);
      bool released = false;
      for (int base = 0; base < total; base += 32 * R) {
        GatherLoader<TILE, R> ld;
        ld.wstage = wstage;
        uint32_t live = 0;
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const int idx = base + i * 32 + lane;
          ld.r[i] = idx < total ? list[idx] : 0;
          if (idx < total) live |= 1u << i;
        }
        if (REL && base + 32 * R >= total) {
          // the tile's last batch: its columns go to registers and the stage goes back
          // before its probes (handing it back after the first probe round, with only the
          // kept rows copied, measured slower: the stage is held through an L2 round trip)
          uint64_t* bar = &empty[s];
          auto give_back = [bar, lane] {
            __syncwarp();
            if (lane == 0) mbar_arrive(bar);
          };
          if (PACK)
            sparse_rows_packed_regs<NSC>(P, ld, live, nd, ns, sparse_bias, A, s_sum, s_touch, smem,
                                         reinterpret_cast<int*>(list), give_back);
          else
            sparse_rows_regs<NSC>(P, ld, live, nd, ns, sparse_bias, A, s_sum, s_touch, smem, give_back);
          released = true;
        } else if (MIR) {
          sparse_rows_mir<NSC>(P, ld, live, nd, ns, sparse_bias, A, s_sum, s_touch, smem);
        } else if (PACK) {
          sparse_rows_packed<NSC>(P, ld, live, nd, ns, sparse_bias, A, s_sum, s_touch, smem);
        } else {
          sparse_rows<NSC, true>(P, ld, live, nd, ns, sparse_bias, A, s_sum, s_touch, smem);
        }
      }
      if (!released) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
      }
      sl += NCW;
      while (sl >= NSL) {
        sl -= NSL;
        next_tile();
      }
    }
    // ---- remainder rows (fewer than one tile per CTA), plain loads -----------------
    if (!failed) {
      const long long tail0 = P.nfull * TILE;
      for (long long r = tail0 + b * (NCW * 32) + (tid - 32); r < P.n; r += G * (NCW * 32)) {
        RowLoader ld{&P, r};
        tail_row(P, ld, A, s_sum, s_touch, smem);
      }
    }
  }

  if (failed) set_status(P.status, MB_STATUS_TIMEOUT);
  if (A.bad_probe) set_status(P.status, MB_STATUS_PROBE_RANGE);
  if (A.bad_group) set_status(P.status, MB_STATUS_GROUP_RANGE);

  // ---- publish -------------------------------------------------------------------
  unsigned long long acc = A.acc, cnt = A.cnt;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc += __shfl_down_sync(kFull, acc, o);
    cnt += __shfl_down_sync(kFull, cnt, o);
  }
  if (lane == 0) {
    s_red[warp] = acc;
    s_red[NWARPS + warp] = cnt;
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
    for (int g = tid; g < P.total_val; g += NWARPS * 32)
      if ((s_touch[g >> 5] >> (g & 31)) & 1u) atomicAdd(group_sum_ptr(P, g), s_sum[g]);
  }
  if (MIR) {
    // no CTA leaves while another may still read its share of the mirrors
    __syncwarp();
    cluster_sync_all();
  }
}

// Variant tables, one per translation unit that instantiates kernels.
const Variant* star_variants_generic(int* count);
const Variant* star_variants_special(int* count);
const Variant* star_variants_wide(int* count);

}  // namespace mb
