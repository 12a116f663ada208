// build.cu — perfect-hash builds over (filtered) dimension tables.
//
//  MB_HT_KEY      atomicCAS(&ht[h], 0, key)                       crystal/join.cuh:167-206
//  MB_HT_KEY_VAL  atomicCAS(&ht[2h], 0, key); ht[2h+1] = val      crystal/join.cuh:236-279
//  MB_HT_VAL_OFF  atomicCAS(&ht[2h], 0, val) if val; ht[2h+1] = row+1
//                                                                 BlockLibrary.cuh:594-715
// with h = (key - key_min) % num_slots (crystal/join.cuh:3). Dimension tables are small
// (<= 1 M rows), so the build is a plain grid-stride kernel; it can also fill a presence
// bitmap that the fused probe stages in shared memory.
#include "common.cuh"
#include "star.cuh"

namespace mb {

__device__ __forceinline__ bool build_pass(int x, int mode, int c1, int c2) {
  if (mode == MB_FILTER_BETWEEN) return x >= c1 && x <= c2;
  if (mode == MB_FILTER_EQ) return x == c1;
  return x == c1 || x == c2;
}

struct BuildPlan {
  const int* filter;   // column / cache-slot index array, or null
  int mode, c1, c2;
  const int* key;
  const int* val;      // or null
  long long n;
  int* ht;
  int slots, kmin, layout;
  uint32_t* presence;
  const int* gpu_cache;
  const short* seg_group;
  long long start_offset;
  int seg_shift;
  unsigned int* status;
  const int* rows;     // optional list of dimension rows to build from (build_GPU3 forms)
  int* min_out;        // optional key range of the rows passing the filter (minmax forms)
  int* max_out;
  int val_min, val_max;  // where each warp's range starts (the reference's block start values)
};

__device__ __forceinline__ long long build_row_index(const BuildPlan& B, long long r, int* seg_out) {
  if (B.rows != nullptr) {
    // a listed dimension row: the physical row, through its own segment's slot
    const long long d = __ldg(B.rows + r);
    if (B.gpu_cache == nullptr) {
      *seg_out = 0;
      return d;
    }
    *seg_out = static_cast<int>(d >> B.seg_shift);
    return d & ((1ll << B.seg_shift) - 1);
  }
  if (B.gpu_cache == nullptr) {
    *seg_out = 0;
    return r;
  }
  const long long vseg = r >> B.seg_shift;
  *seg_out = B.seg_group ? static_cast<int>(B.seg_group[vseg])
                         : static_cast<int>((B.start_offset + r) >> B.seg_shift);
  return r & ((1ll << B.seg_shift) - 1);
}

__device__ __forceinline__ int build_load(const BuildPlan& B, const int* col, int seg, long long idx) {
  if (B.gpu_cache == nullptr) return col[idx];
  return B.gpu_cache[(static_cast<long long>(col[seg]) << B.seg_shift) + idx];
}

__global__ void build_kernel(const __grid_constant__ BuildPlan B) {
  bool bad = false;
  int kmin = B.val_max, kmax = B.val_min;
  for (long long r = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; r < B.n;
       r += static_cast<long long>(gridDim.x) * blockDim.x) {
    int seg;
    const long long idx = build_row_index(B, r, &seg);
    if (B.filter != nullptr && !build_pass(build_load(B, B.filter, seg, idx), B.mode, B.c1, B.c2)) continue;
    const int key = build_load(B, B.key, seg, idx);
    kmin = key < kmin ? key : kmin;
    kmax = key > kmax ? key : kmax;
    const int d = key - B.kmin;
    const int h = (d >= 0 && d < B.slots) ? d : d % B.slots;
    if (h < 0) {
      bad = true;
      continue;
    }
    bool present;
    if (B.layout == MB_HT_KEY) {
      atomicCAS(B.ht + h, 0, key);
      present = key != 0;
    } else if (B.layout == MB_HT_KEY_VAL) {
      const int v = build_load(B, B.val, seg, idx);
      atomicCAS(B.ht + 2ll * h, 0, key);
      B.ht[2ll * h + 1] = v;
      present = key != 0 || v != 0;
    } else {
      // engine layout: the row id is the dimension row's position in the table
      // (segment * segment_size + in-segment offset, or the listed row), stored +1 so 0
      // stays "empty".
      const long long rowid = B.rows != nullptr       ? static_cast<long long>(__ldg(B.rows + r))
                              : B.gpu_cache == nullptr ? B.start_offset + r
                                                       : (static_cast<long long>(seg) << B.seg_shift) + idx;
      if (B.val != nullptr) atomicCAS(B.ht + 2ll * h, 0, build_load(B, B.val, seg, idx));
      B.ht[2ll * h + 1] = static_cast<int>(rowid + 1);
      present = true;
    }
    if (B.presence != nullptr && present) atomicOr(B.presence + (h >> 5), 1u << (h & 31));
  }
  if (bad) set_status(B.status, MB_STATUS_PROBE_RANGE);
  if (B.min_out != nullptr) {
    // every warp folds its range in, starting from (val_max, val_min) as the reference's
    // blocks do (GPUProcessing.h:1052,1101-1110)
    kmin = __reduce_min_sync(0xffffffffu, kmin);
    kmax = __reduce_max_sync(0xffffffffu, kmax);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(B.min_out, kmin);
      atomicMax(B.max_out, kmax);
    }
  }
}

static int launch_build(BuildPlan& B, cudaStream_t stream) {
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  B.status = ds->status;
  if (B.n <= 0) return MB_OK;
  const int threads = 256;
  long long blocks = (B.n + threads - 1) / threads;
  const long long cap = static_cast<long long>(ds->num_sms) * 8;
  if (blocks > cap) blocks = cap;
  build_kernel<<<static_cast<int>(blocks), threads, 0, stream>>>(B);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

}  // namespace mb

using namespace mb;

extern "C" int mb_build_pht(const int* filter_col, int filter_mode, int c1, int c2, const int* dim_key,
                            const int* dim_val, int num_tuples, int* ht, int num_slots, int key_min,
                            uint32_t* presence, mb_stream_t stream) {
  if (num_tuples == 0) return MB_OK;
  if (dim_key == nullptr || ht == nullptr || num_tuples < 0 || num_slots <= 0) return MB_ERR_ARG;
  if (filter_col != nullptr && (filter_mode < MB_FILTER_EQ || filter_mode > MB_FILTER_EQ_OR_EQ)) return MB_ERR_ARG;
  if (dim_val != nullptr && !aligned8(ht)) return MB_ERR_ALIGN;
  BuildPlan B = {};
  B.filter = filter_col;
  B.mode = filter_mode;
  B.c1 = c1;
  B.c2 = c2;
  B.key = dim_key;
  B.val = dim_val;
  B.n = num_tuples;
  B.ht = ht;
  B.slots = num_slots;
  B.kmin = key_min;
  B.layout = dim_val != nullptr ? MB_HT_KEY_VAL : MB_HT_KEY;
  B.presence = presence;
  return launch_build(B, static_cast<cudaStream_t>(stream));
}

extern "C" int mb_join_build(const int* dim_key, const int* dim_val, int num_tuples, int* hash_table,
                             int num_slots, mb_stream_t stream) {
  if (dim_val == nullptr) return MB_ERR_ARG;
  return mb_build_pht(nullptr, 0, 0, 0, dim_key, dim_val, num_tuples, hash_table, num_slots, 0, nullptr, stream);
}

// The engine builds (VAL_OFF layout): build_GPU2 / build_GPU_minmax over a segment range,
// build_GPU3 / build_GPU_minmax2 over a list of dimension rows (dim_off), the minmax forms
// also folding the key range into *min_out / *max_out.
static int engine_build(const int* gpuCache, const int* dim_off, const mb_filterArgsGPU* fargs,
                        const mb_buildArgsGPU* bargs, int num_tuples, int* hash_table, int start_offset,
                        const short* segment_group, int* min_out, int* max_out, mb_stream_t stream) {
  if (num_tuples == 0) return MB_OK;
  if (bargs == nullptr || bargs->key_idx == nullptr || hash_table == nullptr || num_tuples < 0 ||
      bargs->num_slots <= 0)
    return MB_ERR_ARG;
  if ((min_out == nullptr) != (max_out == nullptr)) return MB_ERR_ARG;
  if (!aligned8(hash_table)) return MB_ERR_ALIGN;
  // the list forms take no filter (GPUProcessing.h:1018, cudaAssert(fargs.filter_idx1 == NULL))
  if (dim_off != nullptr && fargs != nullptr && fargs->filter_idx1 != nullptr) return MB_ERR_ARG;
  BuildPlan B = {};
  B.rows = dim_off;
  B.min_out = min_out;
  B.max_out = max_out;
  B.val_min = bargs->val_min;
  B.val_max = bargs->val_max;
  if (fargs != nullptr && fargs->filter_idx1 != nullptr) {
    if (fargs->mode1 < MB_FILTER_EQ || fargs->mode1 > MB_FILTER_EQ_OR_EQ) return MB_ERR_ARG;
    B.filter = fargs->filter_idx1;
    B.mode = fargs->mode1;
    B.c1 = fargs->compare1;
    B.c2 = fargs->compare2;
  }
  B.key = bargs->key_idx;
  B.val = bargs->val_idx;
  B.n = num_tuples;
  B.ht = hash_table;
  B.slots = bargs->num_slots;
  B.kmin = bargs->val_min;
  B.layout = MB_HT_VAL_OFF;
  B.gpu_cache = gpuCache;
  B.seg_group = dim_off != nullptr ? nullptr : segment_group;
  B.start_offset = dim_off != nullptr ? 0 : start_offset;
  B.seg_shift = 20;  // SEGMENT_SIZE = 1,048,576 (src/gpudb/common.h:73)
  return launch_build(B, static_cast<cudaStream_t>(stream));
}

extern "C" int mb_build_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_buildArgsGPU* bargs,
                             int num_tuples, int* hash_table, int start_offset, const short* segment_group,
                             mb_stream_t stream) {
  return engine_build(gpuCache, nullptr, fargs, bargs, num_tuples, hash_table, start_offset, segment_group, nullptr,
                      nullptr, stream);
}

extern "C" int mb_build_GPU3(const int* gpuCache, const int* dim_off, const mb_filterArgsGPU* fargs,
                             const mb_buildArgsGPU* bargs, int num_tuples, int* hash_table, mb_stream_t stream) {
  if (dim_off == nullptr) return MB_ERR_ARG;
  return engine_build(gpuCache, dim_off, fargs, bargs, num_tuples, hash_table, 0, nullptr, nullptr, nullptr, stream);
}

extern "C" int mb_build_GPU_minmax(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_buildArgsGPU* bargs,
                                   int num_tuples, int* hash_table, int* min_global, int* max_global,
                                   int start_offset, const short* segment_group, mb_stream_t stream) {
  if (min_global == nullptr || max_global == nullptr) return MB_ERR_ARG;
  return engine_build(gpuCache, nullptr, fargs, bargs, num_tuples, hash_table, start_offset, segment_group,
                      min_global, max_global, stream);
}

extern "C" int mb_build_GPU_minmax2(const int* gpuCache, const int* dim_off, const mb_filterArgsGPU* fargs,
                                    const mb_buildArgsGPU* bargs, int num_tuples, int* hash_table, int* min_global,
                                    int* max_global, mb_stream_t stream) {
  if (dim_off == nullptr || min_global == nullptr || max_global == nullptr) return MB_ERR_ARG;
  return engine_build(gpuCache, dim_off, fargs, bargs, num_tuples, hash_table, 0, nullptr, min_global, max_global,
                      stream);
}
