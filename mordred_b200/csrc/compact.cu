// compact.cu — selection with compaction: the rows of a fact range (or of an input
// offset list) that pass a query's filters and probes, written out as an offset list of
// physical rows plus, per probe, the dimension offset or payload the probe found.
//
// This is the handoff of CPU/GPU split execution: when a query's filters and probes run
// on the GPU but its aggregation runs on the CPU (or the other way round), the survivors
// cross PCIe as offset lists (src/gpudb/CPUGPUProcessing.cu:60-144 switch_device_fact).
// Restates the reference's compaction kernels filter_GPU2/3, filter_probe_GPU2/3 and
// probe_GPU2/3 (src/gpudb/GPUProcessing.h:496-925, 1174-1383), which scan per block and
// take one atomicAdd on the output cursor per block; here each warp ballots its 32 rows
// and takes one atomicAdd per warp, so the list order is not deterministic (it never is
// in the reference either) while its set of rows is.
//
// Probe outputs per layout: MB_HT_VAL_OFF (engine builds) — present when the row word
// ht[2h+1] != 0, output ht[2h+1] - 1, the dimension row (BlockLibrary.cuh:9-33);
// MB_HT_KEY_VAL — present when the 8-byte slot != 0, output the payload; MB_HT_KEY —
// present when ht[h] != 0, output 0.
#include "common.cuh"

namespace mb {

struct SelPlan {
  long long n;               // virtual rows, or entries of in_rows
  const int* in_rows;        // physical-row input list (list form), or null
  const int* in_dim[4];      // list form: dimension offsets passed through to dim slots not probed here
  int nf;
  const int* fcol[MB_MAX_FILTERS];
  int fmode[MB_MAX_FILTERS], fc1[MB_MAX_FILTERS], fc2[MB_MAX_FILTERS];
  int np;
  const int* pkey[MB_MAX_PROBES];
  const int* pht[MB_MAX_PROBES];
  int pslots[MB_MAX_PROBES], pkmin[MB_MAX_PROBES], playout[MB_MAX_PROBES];
  int slot_src[4];           // output dim slot j <- probe index, or -1: pass in_dim[j] through
  int* dim_out[4];
  int* lo_off;
  int* total;
  long long capacity;        // entries the output lists hold
  const int* gpu_cache;      // segment addressing (column fields are slot-index arrays)
  const short* seg_group;
  long long start_offset;
  int seg_shift;
  unsigned int* status;
};

__device__ __forceinline__ bool sel_pass(int x, int mode, int c1, int c2) {
  return mode == MB_FILTER_BETWEEN ? (x >= c1 && x <= c2) : mode == MB_FILTER_EQ ? x == c1 : (x == c1 || x == c2);
}

template <int ITEMS>
__global__ void __launch_bounds__(256) select_kernel(const __grid_constant__ SelPlan P) {
  const int lane = threadIdx.x & 31;
  const long long gwarp = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  const long long S = 1ll << P.seg_shift;
  bool bad_probe = false, overflow = false;
  for (long long base = gwarp * 32 * ITEMS; base < P.n; base += nwarps * 32 * ITEMS) {
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
      const long long i = base + it * 32 + lane;
      bool ok = i < P.n;
      long long phys = 0, idx = 0;  // physical row; column index (plain) or in-segment offset
      int seg = 0;
      if (ok) {
        if (P.in_rows) {
          phys = P.in_rows[i];
        } else if (P.gpu_cache && P.seg_group) {
          phys = (static_cast<long long>(P.seg_group[i >> P.seg_shift]) << P.seg_shift) + (i & (S - 1));
        } else {
          phys = P.start_offset + i;
        }
        if (P.gpu_cache) {
          seg = static_cast<int>(phys >> P.seg_shift);
          idx = phys & (S - 1);
        } else {
          idx = phys - P.start_offset;
        }
      }
      auto load = [&](const int* col) -> int {
        if (P.gpu_cache) return __ldg(P.gpu_cache + (static_cast<long long>(__ldg(col + seg)) << P.seg_shift) + idx);
        return __ldg(col + idx);
      };
      for (int f = 0; f < P.nf; ++f)
        if (ok) ok = sel_pass(load(P.fcol[f]), P.fmode[f], P.fc1[f], P.fc2[f]);
      int outv[MB_MAX_PROBES] = {0, 0, 0, 0};
      for (int p = 0; p < P.np; ++p) {
        if (!ok) break;
        const int h = pht_slot(load(P.pkey[p]), P.pslots[p], P.pkmin[p]);
        if (h < 0) {
          bad_probe = true;
          ok = false;
          break;
        }
        const int* ht = P.pht[p];
        if (P.playout[p] == MB_HT_KEY) {
          ok = __ldg(ht + h) != 0;
        } else if (P.playout[p] == MB_HT_VAL_OFF) {
          const int w = __ldg(ht + 2ll * h + 1);
          ok = w != 0;
          outv[p] = w - 1;
        } else {
          const unsigned long long s = ldg_u64(ht + 2ll * h);
          ok = s != 0;
          outv[p] = static_cast<int>(s >> 32);
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, ok);
      if (m == 0) continue;
      int b0 = 0;
      if (lane == 0) b0 = atomicAdd(P.total, __popc(m));
      b0 = __shfl_sync(0xffffffffu, b0, 0);
      if (!ok) continue;
      const long long pos = static_cast<long long>(b0) + __popc(m & ((1u << lane) - 1u));
      if (pos >= P.capacity) {
        overflow = true;
        continue;
      }
      P.lo_off[pos] = static_cast<int>(phys);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (P.dim_out[j] == nullptr) continue;
        const int src = P.slot_src[j];
        P.dim_out[j][pos] = src >= 0 ? outv[src] : (P.in_dim[j] ? P.in_dim[j][i] : 0);
      }
    }
  }
  if (bad_probe) set_status(P.status, MB_STATUS_PROBE_RANGE);
  if (overflow) set_status(P.status, MB_STATUS_OVERFLOW);
}

static int launch_select(SelPlan& P, cudaStream_t st) {
  if (P.n == 0) return MB_OK;
  if (P.n < 0 || P.lo_off == nullptr || P.total == nullptr || P.capacity < 0) return MB_ERR_ARG;
  if (P.gpu_cache == nullptr && P.seg_group != nullptr) return MB_ERR_ARG;
  for (int f = 0; f < P.nf; ++f)
    if (P.fcol[f] == nullptr || P.fmode[f] < MB_FILTER_EQ || P.fmode[f] > MB_FILTER_EQ_OR_EQ) return MB_ERR_ARG;
  for (int p = 0; p < P.np; ++p) {
    if (P.pkey[p] == nullptr || P.pht[p] == nullptr || P.pslots[p] <= 0) return MB_ERR_ARG;
    if (P.playout[p] < MB_HT_KEY || P.playout[p] > MB_HT_VAL_OFF) return MB_ERR_ARG;
    if (P.playout[p] != MB_HT_KEY && !aligned8(P.pht[p])) return MB_ERR_ALIGN;
  }
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  P.status = ds->status;
  constexpr int kItems = 4, kThreads = 256;
  const long long per_block = static_cast<long long>(kThreads) * kItems;
  long long blocks = (P.n + per_block - 1) / per_block;
  if (blocks > static_cast<long long>(ds->num_sms) * 8) blocks = static_cast<long long>(ds->num_sms) * 8;
  select_kernel<kItems><<<static_cast<int>(blocks), kThreads, 0, st>>>(P);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

static void engine_filters(SelPlan& P, const mb_filterArgsGPU* f) {
  if (f == nullptr) return;
  if (f->filter_idx1) {
    P.fcol[P.nf] = f->filter_idx1;
    P.fmode[P.nf] = f->mode1;
    P.fc1[P.nf] = f->compare1;
    P.fc2[P.nf++] = f->compare2;
  }
  if (f->filter_idx2) {
    P.fcol[P.nf] = f->filter_idx2;
    P.fmode[P.nf] = f->mode2;
    P.fc1[P.nf] = f->compare3;
    P.fc2[P.nf++] = f->compare4;
  }
}

// Engine probes, dimension slots 1..4 = supplier, customer, part, date, over VAL_OFF tables.
static void engine_probes(SelPlan& P, const mb_probeArgsGPU* q) {
  for (int j = 0; j < 4; ++j) P.slot_src[j] = -1;
  if (q == nullptr) return;
  const int* keys[4] = {q->key_idx1, q->key_idx2, q->key_idx3, q->key_idx4};
  const int* hts[4] = {q->ht1, q->ht2, q->ht3, q->ht4};
  const int lens[4] = {q->dim_len1, q->dim_len2, q->dim_len3, q->dim_len4};
  const int mins[4] = {q->min_key1, q->min_key2, q->min_key3, q->min_key4};
  for (int j = 0; j < 4; ++j) {
    if (keys[j] == nullptr || hts[j] == nullptr) continue;
    P.pkey[P.np] = keys[j];
    P.pht[P.np] = hts[j];
    P.pslots[P.np] = lens[j];
    P.pkmin[P.np] = mins[j];
    P.playout[P.np] = MB_HT_VAL_OFF;
    P.slot_src[j] = P.np++;
  }
}

static void engine_out(SelPlan& P, const mb_offsetGPU* out, const mb_offsetGPU* in) {
  P.lo_off = out ? out->lo_off : nullptr;
  int* const outs[4] = {out ? out->dim_off1 : nullptr, out ? out->dim_off2 : nullptr, out ? out->dim_off3 : nullptr,
                        out ? out->dim_off4 : nullptr};
  const int* const ins[4] = {in ? in->dim_off1 : nullptr, in ? in->dim_off2 : nullptr, in ? in->dim_off3 : nullptr,
                             in ? in->dim_off4 : nullptr};
  for (int j = 0; j < 4; ++j) {
    P.dim_out[j] = outs[j];
    P.in_dim[j] = ins[j];
  }
}

static int engine_select(const int* gpuCache, const mb_offsetGPU* in_off, const mb_filterArgsGPU* f,
                         const mb_probeArgsGPU* q, const mb_offsetGPU* out_off, int num_tuples, int* total,
                         int start_offset, const short* segment_group, cudaStream_t st) {
  if (num_tuples == 0) return MB_OK;
  if (gpuCache == nullptr || out_off == nullptr || num_tuples < 0) return MB_ERR_ARG;
  if (in_off != nullptr && in_off->lo_off == nullptr) return MB_ERR_ARG;
  SelPlan P = {};
  P.n = num_tuples;
  P.in_rows = in_off ? in_off->lo_off : nullptr;
  engine_filters(P, f);
  engine_probes(P, q);
  engine_out(P, out_off, in_off);
  P.capacity = num_tuples;
  P.total = total;
  P.gpu_cache = gpuCache;
  P.seg_group = in_off ? nullptr : segment_group;
  P.start_offset = in_off ? 0 : start_offset;
  P.seg_shift = 20;  // SEGMENT_SIZE = 1,048,576 (src/gpudb/common.h:73)
  return launch_select(P, st);
}

}  // namespace mb

using namespace mb;

extern "C" int mb_star_select(const mb_star_args* a, const int* in_rows, int64_t num_in, int* lo_off,
                              int* const* dim_off, int64_t capacity, int* total, mb_stream_t stream) {
  if (a == nullptr) return MB_ERR_ARG;
  if (a->num_filters < 0 || a->num_filters > MB_MAX_FILTERS || a->num_probes < 0 || a->num_probes > MB_MAX_PROBES)
    return MB_ERR_ARG;
  SelPlan P = {};
  P.n = in_rows ? num_in : a->num_rows;
  P.in_rows = in_rows;
  P.nf = a->num_filters;
  for (int f = 0; f < P.nf; ++f) {
    P.fcol[f] = a->filter[f].col;
    P.fmode[f] = a->filter[f].mode;
    P.fc1[f] = a->filter[f].c1;
    P.fc2[f] = a->filter[f].c2;
  }
  P.np = a->num_probes;
  for (int p = 0; p < 4; ++p) P.slot_src[p] = p < P.np ? p : -1;
  for (int p = 0; p < P.np; ++p) {
    P.pkey[p] = a->probe[p].fkey;
    P.pht[p] = a->probe[p].ht;
    P.pslots[p] = a->probe[p].num_slots;
    P.pkmin[p] = a->probe[p].key_min;
    P.playout[p] = a->probe[p].layout;
    P.dim_out[p] = dim_off ? dim_off[p] : nullptr;
  }
  P.lo_off = lo_off;
  P.total = total;
  P.capacity = capacity;
  P.gpu_cache = a->gpu_cache;
  P.seg_group = a->gpu_cache ? a->segment_group : nullptr;
  P.start_offset = a->start_offset;
  if (a->gpu_cache) {
    if (a->segment_size <= 0 || (a->segment_size & (a->segment_size - 1)) != 0) return MB_ERR_ARG;
    P.seg_shift = __builtin_ctz(static_cast<unsigned>(a->segment_size));
  }
  return launch_select(P, static_cast<cudaStream_t>(stream));
}

extern "C" int mb_filter_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_offsetGPU* out_off,
                              int num_tuples, int* total, int start_offset, const short* segment_group,
                              mb_stream_t stream) {
  return engine_select(gpuCache, nullptr, fargs, nullptr, out_off, num_tuples, total, start_offset, segment_group,
                       static_cast<cudaStream_t>(stream));
}

extern "C" int mb_filter_probe_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs,
                                    const mb_probeArgsGPU* pargs, const mb_offsetGPU* out_off, int num_tuples,
                                    int* total, int start_offset, const short* segment_group, mb_stream_t stream) {
  return engine_select(gpuCache, nullptr, fargs, pargs, out_off, num_tuples, total, start_offset, segment_group,
                       static_cast<cudaStream_t>(stream));
}

extern "C" int mb_probe_GPU2(const int* gpuCache, const mb_probeArgsGPU* pargs, const mb_offsetGPU* out_off,
                             int num_tuples, int* total, int start_offset, const short* segment_group,
                             mb_stream_t stream) {
  return engine_select(gpuCache, nullptr, nullptr, pargs, out_off, num_tuples, total, start_offset, segment_group,
                       static_cast<cudaStream_t>(stream));
}

extern "C" int mb_filter_GPU3(const int* gpuCache, const mb_offsetGPU* in_off, const mb_filterArgsGPU* fargs,
                              const mb_offsetGPU* out_off, int num_tuples, int* total, mb_stream_t stream) {
  return engine_select(gpuCache, in_off, fargs, nullptr, out_off, num_tuples, total, 0, nullptr,
                       static_cast<cudaStream_t>(stream));
}

extern "C" int mb_filter_probe_GPU3(const int* gpuCache, const mb_offsetGPU* in_off, const mb_filterArgsGPU* fargs,
                                    const mb_probeArgsGPU* pargs, const mb_offsetGPU* out_off, int num_tuples,
                                    int* total, mb_stream_t stream) {
  return engine_select(gpuCache, in_off, fargs, pargs, out_off, num_tuples, total, 0, nullptr,
                       static_cast<cudaStream_t>(stream));
}

extern "C" int mb_probe_GPU3(const int* gpuCache, const mb_offsetGPU* in_off, const mb_probeArgsGPU* pargs,
                             const mb_offsetGPU* out_off, int num_tuples, int* total, mb_stream_t stream) {
  return engine_select(gpuCache, in_off, nullptr, pargs, out_off, num_tuples, total, 0, nullptr,
                       static_cast<cudaStream_t>(stream));
}
