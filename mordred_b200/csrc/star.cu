// star.cu — host launcher of the fused star-query kernel and its generic variants
// (shape read from the plan at run time). Device code: star_impl.cuh.
#include <climits>
#include <cstring>

#include "star_impl.cuh"
#include "tuned_configs.h"

namespace mb {

static const Variant kGeneric[] = {
    {4, 4, -1, -1, -1, star_kernel<4, 4, -1, -1, -1>},    {4, 8, -1, -1, -1, star_kernel<4, 8, -1, -1, -1>},
    {4, 16, -1, -1, -1, star_kernel<4, 16, -1, -1, -1>},  {8, 4, -1, -1, -1, star_kernel<8, 4, -1, -1, -1>},
    {8, 8, -1, -1, -1, star_kernel<8, 8, -1, -1, -1>},    {8, 16, -1, -1, -1, star_kernel<8, 16, -1, -1, -1>},
    {16, 4, -1, -1, -1, star_kernel<16, 4, -1, -1, -1>},  {16, 8, -1, -1, -1, star_kernel<16, 8, -1, -1, -1>},
    {16, 16, -1, -1, -1, star_kernel<16, 16, -1, -1, -1>},
};

const Variant* star_variants_generic(int* count) {
  *count = static_cast<int>(sizeof(kGeneric) / sizeof(kGeneric[0]));
  return kGeneric;
}

// The specialised variant for this shape if one was compiled, else the generic one. The
// mirror-reading variants exist for specialised shapes only.
static const Variant* find_variant(int warps, int items, int nf, int nd, int ns, bool mir, bool pack = false,
                                   bool rel = false) {
  int n = 0;
  for (int t = 0; t < 2; ++t) {
    const Variant* sp = t == 0 ? star_variants_special(&n) : star_variants_wide(&n);
    for (int i = 0; i < n; ++i)
      if (sp[i].warps == warps && sp[i].items == items && sp[i].nf == nf && sp[i].nd == nd && sp[i].ns == ns &&
          sp[i].mir == mir && sp[i].pack == pack && sp[i].rel == rel)
        return &sp[i];
  }
  if (mir) return nullptr;
  if (rel) return find_variant(warps, items, nf, nd, ns, false, pack, false);  // no early-return variant
  if (pack) return find_variant(warps, items, nf, nd, ns, false, false);  // no packing variant: plain one
  const Variant* g = star_variants_generic(&n);
  for (int i = 0; i < n; ++i)
    if (g[i].warps == warps && g[i].items == items) return &g[i];
  return nullptr;
}

int star_init_device(const DeviceState& ds) {
  for (int t = 0; t < 3; ++t) {
    int n = 0;
    const Variant* v = t == 0 ? star_variants_generic(&n) : t == 1 ? star_variants_special(&n) : star_variants_wide(&n);
    for (int i = 0; i < n; ++i) {
      cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(v[i].fn),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, ds.max_smem_optin - 2048);
      if (e != cudaSuccess) return MB_ERR_CUDA;
    }
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

// Lay out shared memory for `stages` stages; returns total bytes. A mirror share (P.cluster >
// 1) sits between the survivor lists and the stage ring.
static int layout_smem(StarPlan& P, int ncw, int items, int stages, bool stage_bitmaps, bool xfer) {
  const int tile = tile_slices(ncw) * 32 * items;
  int off = 3 * kMaxStages * 8;  // full (two per stage) and empty mbarriers
  P.smem_groups_off = off;
  if (P.gmode == kGroupSmem) off += round_up(8 * P.total_val + 4 * ((P.total_val + 31) / 32), 128);
  int bm_total = 0;
  P.n_dense = 0;
  P.sparse_p0 = 0;
  P.dense_bias = 0;
  bool leading = true, payload_free = true;
  for (int p = 0; p < P.np; ++p) {
    P.p_bm_off[p] = -1;
    P.p_bm_words[p] = 0;
    const int words = (P.p_slots[p] + 31) / 32;
    // a presence bitmap comes from the caller, or the kernel derives it from the table:
    // any MB_HT_KEY table (its test replaces the table load), and a small table with
    // 8-byte slots when it leads the chain (its test then filters in the dense phase)
    const bool have = P.p_presence[p] != nullptr || P.p_layout[p] == MB_HT_KEY ||
                      (leading && P.p_slots[p] <= kBitmapDeriveMaxSlots8);
    if (stage_bitmaps && have && words * 4 <= kBitmapSmemMaxBytes && bm_total + words * 4 <= kBitmapSmemTotalBytes) {
      P.p_bm_off[p] = off;
      P.p_bm_words[p] = words;
      off += round_up(words * 4, 16);
      bm_total += words * 4;
    }
    // leading probes with a staged bitmap are tested in the dense phase. One whose
    // payload nobody reads (an MB_HT_KEY table, or a zero group multiplier with the
    // payload not stored) is settled there: its group term is the constant
    // (0 - min_val) * unique_val. The others are probed again in the sparse phase, for
    // the survivors only, to read their payloads.
    if (leading && P.p_bm_off[p] >= 0) {
      P.n_dense = p + 1;
      // (MB_AGG_MUL_PAYLOAD multiplies by the first probe's payload: that one is never free)
      const bool free = (P.p_layout[p] == MB_HT_KEY || (P.p_mul[p] == 0 && P.p_res_slot[p] < 0)) &&
                        !(p == 0 && P.agg_op == MB_AGG_MUL_PAYLOAD);
      if (payload_free && free) {
        P.sparse_p0 = p + 1;
        P.dense_bias += (0u - static_cast<unsigned>(P.p_min[p])) * static_cast<unsigned>(P.p_mul[p]);
      } else {
        payload_free = false;
      }
    } else {
      leading = false;
    }
  }
  off = round_up(off, 16);
  P.smem_list_off = off;
  off += ncw * star_list_bytes(items, xfer);
  off = round_up(off, 16);
  P.smem_mirror_off = off;
  if (P.cluster > 1) off += 4 << P.mir_shift;
  off = round_up(off, 128);
  P.smem_stage_off = off;
  P.stage_bytes = P.ncols * tile * 4;
  P.stages = stages;
  P.smem_total = off + stages * P.stage_bytes;
  return P.smem_total;
}

// Plan cluster-resident mirrors for the sparse phase's table probes (those without a staged
// bitmap): presence bits, or 4-bit payload codes when the probe's payload is read and its
// group term leaves at most 14 payload values (the next larger group multiplier, or the
// group count, over its own). Chooses the cluster size and the per-CTA share; returns false
// (and clears the plan) when no probe qualifies or the mirrors do not fit.
static bool plan_mirrors(StarPlan& P) {
  P.cluster = 1;
  P.mir_shift = 0;
  long long words = 0;
  bool any = false;
  for (int p = 0; p < P.np; ++p) {
    P.mir_kind[p] = kMirNone;
    P.mir_base[p] = P.mir_words[p] = P.mir_min[p] = P.mir_payload[p] = 0;
  }
  for (int p = P.sparse_p0; p < P.np; ++p) {
    if (P.p_bm_off[p] >= 0) continue;  // probed against its staged bitmap already
    const bool need = !(P.p_layout[p] == MB_HT_KEY || (P.p_mul[p] == 0 && P.p_res_slot[p] < 0)) ||
                      (p == 0 && P.agg_op == MB_AGG_MUL_PAYLOAD);
    int kind = kMirBits;
    if (need && P.p_layout[p] != MB_HT_KEY) {
      // payload values the group term can tell apart: next multiplier above this one's, over it
      long long next = P.gmode == kGroupScalar ? 1 : P.total_val;
      for (int o = 0; o < P.np; ++o)
        if (o != p && P.p_mul[o] > P.p_mul[p] && P.p_mul[o] < next) next = P.p_mul[o];
      if (P.p_mul[p] > 0 && P.p_res_slot[p] >= 0 && next / P.p_mul[p] <= 14) kind = kMirNibble;
    }
    const long long w = kind == kMirNibble ? (P.p_slots[p] + 7ll) / 8 : (P.p_slots[p] + 31ll) / 32;
    if (words + w > static_cast<long long>(kMirrorMaxCluster) * kMirrorMaxShareWords) continue;
    P.mir_kind[p] = kind;
    P.mir_base[p] = static_cast<int>(words);
    P.mir_words[p] = static_cast<int>(w);
    P.mir_min[p] = P.p_min[p];
    P.mir_payload[p] = need ? 1 : 0;
    words += w;
    any = true;
  }
  if (!any) return false;
  // the smallest share that fits with the portable cluster size, clusters of 8 (shares of
  // at most kMirrorMaxShareWords); smaller shares leave more shared memory for stages
  int shift = 0;
  while ((static_cast<long long>(kMirrorMaxCluster) << shift) < words) ++shift;
  P.cluster = kMirrorMaxCluster;
  P.mir_shift = shift;
  return true;
}

static void clear_mirrors(StarPlan& P) {
  P.cluster = 1;
  P.mir_shift = 0;
  for (int p = 0; p < MB_MAX_PROBES; ++p) P.mir_kind[p] = kMirNone;
}

int launch_star(const mb_star_args* a, cudaStream_t stream, int count32, const DeviceState* preset) {
  if (a == nullptr) return MB_ERR_ARG;
  if (a->num_rows < 0) return MB_ERR_ARG;
  if (a->num_rows == 0) return MB_OK;  // empty input: nothing to add (pointers may be null)
  if (a->num_filters < 0 || a->num_filters > MB_MAX_FILTERS) return MB_ERR_ARG;
  if (a->num_probes < 0 || a->num_probes > MB_MAX_PROBES) return MB_ERR_ARG;
  if (a->aggr[0] == nullptr) return MB_ERR_ARG;
  if (a->agg_op < MB_AGG_SUM || a->agg_op > MB_AGG_MUL_PAYLOAD) return MB_ERR_ARG;
  const bool two_cols = a->agg_op == MB_AGG_SUB || a->agg_op == MB_AGG_MUL;
  if (two_cols && a->aggr[1] == nullptr) return MB_ERR_ARG;
  if (a->agg_op == MB_AGG_MUL_PAYLOAD && (a->num_probes < 1 || a->probe[0].layout == MB_HT_KEY)) return MB_ERR_ARG;
  if (a->res == nullptr) return MB_ERR_ARG;
  if (!aligned8(a->res)) return MB_ERR_ALIGN;
  if (a->res_layout < MB_RES_SCALAR || a->res_layout > MB_RES_DENSE) return MB_ERR_ARG;
  if (a->res_layout != MB_RES_SCALAR && a->total_val <= 0) return MB_ERR_ARG;
  if (a->count != nullptr && !count32 && !aligned8(a->count)) return MB_ERR_ALIGN;
  if (a->group_mode < 0 || a->group_mode > 2) return MB_ERR_ARG;

  int err = MB_OK;
  const DeviceState* ds = preset != nullptr ? preset : current_device_state(&err);
  if (ds == nullptr) return err;

  // an offset-list input, or a group value passed through from an earlier join, runs the
  // gather form of the pipeline
  bool list_form = a->rows != nullptr;
  for (int p = 0; p < a->num_probes; ++p) list_form = list_form || a->probe[p].layout == MB_HT_PASS;
  if (list_form) {
    if (count32) return MB_ERR_ARG;
    return launch_list(a, stream, ds);
  }

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

  // ---- launch configuration and shared-memory plan ------------------------------
  // Unset fields take the tuned configuration for this query shape (tuned_configs.h).
  const TunedConfig tc = tuned_config(P.nf, a->num_probes, a->probe[0].layout, P.res_layout, P.total_val, P.n);
  const int threads = a->threads ? a->threads : tc.threads;
  const int items = a->items_per_thread ? a->items_per_thread : tc.items;
  if (threads % 32 != 0 || threads < 128 || threads > 768) return MB_ERR_ARG;
  if (items != 4 && items != 8 && items != 16) return MB_ERR_ARG;
  const int ncw = threads / 32;
  const int tile = tile_slices(ncw) * 32 * items;
  if (P.gpu_cache != nullptr && (1 << P.seg_shift) < tile) return MB_ERR_ARG;

  bool direct_aligned = true;
  for (int c = 0; c < P.ncols; ++c) direct_aligned = direct_aligned && aligned16(P.col[c]);
  const bool use_tiles = P.gpu_cache != nullptr || direct_aligned;
  P.nfull = use_tiles ? P.n / tile : 0;

  const int group_mode = a->group_mode ? a->group_mode : tc.group_mode;
  if (P.res_layout == MB_RES_SCALAR)
    P.gmode = kGroupScalar;
  else if (group_mode == 2)
    P.gmode = kGroupGlobal;
  else
    P.gmode = P.total_val <= kSmemGroupMax ? kGroupSmem : kGroupGlobal;
  if (group_mode == 1 && P.gmode != kGroupSmem) return MB_ERR_SIZE;

  if (a->mirrors < 0 || a->mirrors > 2) return MB_ERR_ARG;
  if (a->pack < 0 || a->pack > 4) return MB_ERR_ARG;
  const bool want_pack = a->pack == 2 || a->pack == 3 || (a->pack == 0 && (tc.pack == 1 || tc.pack == 2));
  const bool want_rel = a->pack >= 3 || (a->pack == 0 && tc.pack >= 2);
  const int budget = ds->max_smem_optin - 2048 - 2 * 8 * (ncw + 1);
  const int want_stages = a->stages ? a->stages : tc.stages;
  if (want_stages < 2 || want_stages > kMaxStages) return MB_ERR_ARG;
  clear_mirrors(P);
  const bool xfer = want_pack && want_rel;  // the survivor lists double as the packing buffer
  auto fit = [&]() -> int {
    int smem = layout_smem(P, ncw, items, want_stages, true, xfer);
    while (smem > budget && P.stages > 2) smem = layout_smem(P, ncw, items, P.stages - 1, true, xfer);
    if (smem > budget && P.gmode == kGroupSmem && group_mode != 1) {
      P.gmode = kGroupGlobal;
      smem = layout_smem(P, ncw, items, want_stages, true, xfer);
      while (smem > budget && P.stages > 2) smem = layout_smem(P, ncw, items, P.stages - 1, true, xfer);
    }
    return smem;
  };
  int smem = fit();
  // cluster-resident mirrors: on request (mirrors = 2), or by default for large calls with
  // tiles; the plan needs the staged bitmaps laid out first, then the layout is redone
  // with the mirror share
  const bool try_mir = use_tiles && P.nfull > 0 && a->mirrors != 1 &&
                       (a->mirrors == 2 || (tc.mirrors && P.n >= kMirrorMinRows)) && preset == nullptr;
  const Variant* var = nullptr;
  if (try_mir && smem <= budget && plan_mirrors(P)) {
    const GroupMode keep_gmode = static_cast<GroupMode>(P.gmode);
    smem = fit();
    var = smem <= budget ? find_variant(ncw, items, P.nf, P.n_dense, P.np - P.sparse_p0, true) : nullptr;
    if (var == nullptr) {
      clear_mirrors(P);
      P.gmode = keep_gmode;
      smem = fit();
    }
  }
  if (smem > budget) smem = layout_smem(P, ncw, items, 2, false, xfer);
  if (smem > budget) return MB_ERR_SIZE;
  if (var == nullptr)
    var = find_variant(ncw, items, P.nf, P.n_dense, P.np - P.sparse_p0, false, want_pack, want_rel);
  if (var == nullptr && ncw > kMaxTileSlices) {
    // wide launches (more consumer warps than tile slices) are compiled for the packed
    // shapes only; a call whose plan lands on another shape — small dimension tables
    // that get a staged bitmap and join the dense phase, or misaligned columns that
    // leave only the per-row path — takes 16 consumer warps
    mb_star_args narrow = *a;
    narrow.threads = kMaxTileSlices * 32;
    return launch_star(&narrow, stream, count32, preset);
  }
  if (var == nullptr) return MB_ERR_ARG;

  // sparse visiting order of the tiled path: chain order, except that the first probe
  // the dense phase did not settle goes first (a settled probe is present for every row
  // the dense phase passes, so reading its payload later changes no result or status
  // bit). The mirror-reading sparse phase and a payload-multiplied aggregate (which reads
  // the first probe's payload) keep chain order.
  const int ns_total = P.np - P.sparse_p0;
  for (int q = 0; q < ns_total; ++q) P.sp_ord[q] = P.sparse_p0 + q;
  if (!var->mir && P.agg_op != MB_AGG_MUL_PAYLOAD) {
    const int first = P.n_dense - P.sparse_p0;
    if (first > 0 && first < ns_total) {
      const int lead = P.sp_ord[first];
      for (int q = first; q > 0; --q) P.sp_ord[q] = P.sp_ord[q - 1];
      P.sp_ord[0] = lead;
    }
  }

  long long want = P.nfull > 0 ? P.nfull : (P.n + threads - 1) / threads;
  if (want < 1) want = 1;
  if (var->mir) {
    // one cluster of P.cluster CTAs per group of SMs; every CTA of a cluster holds a share
    // of the mirrors, so the grid is whole clusters (CTAs without tiles still hold one)
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(P.cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(threads + 32);
    cfg.dynamicSmemBytes = static_cast<size_t>(smem);
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = a->grid > 0 ? (a->grid + P.cluster - 1) / P.cluster : 0;
    if (clusters <= 0) {
      cfg.gridDim = dim3(static_cast<unsigned>(P.cluster * 64));
      if (cudaOccupancyMaxActiveClusters(&clusters, reinterpret_cast<const void*>(var->fn), &cfg) != cudaSuccess)
        return MB_ERR_CUDA;
      if (clusters < 1) return MB_ERR_SIZE;
    }
    const long long need_clusters = (want + P.cluster - 1) / P.cluster;
    if (clusters > need_clusters) clusters = static_cast<int>(need_clusters);
    cfg.gridDim = dim3(static_cast<unsigned>(clusters * P.cluster));
    if (cudaLaunchKernelEx(&cfg, var->fn, P) != cudaSuccess) return MB_ERR_LAUNCH;
    note_launches(1);
    return MB_OK;
  }

  int grid = a->grid;
  if (grid <= 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, var->fn, threads + 32, smem) != cudaSuccess)
      return MB_ERR_CUDA;
    if (per_sm < 1) per_sm = 1;
    grid = ds->num_sms * per_sm;
  }
  if (grid > want) grid = static_cast<int>(want);

  var->fn<<<grid, threads + 32, smem, stream>>>(P);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

}  // namespace mb
