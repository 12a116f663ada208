// segcache.cpp — the GPU segment cache: fact columns split into fixed-size segments,
// a pool of segment slots in device memory, a (column, segment) -> slot map, and the
// admission / replacement policies that decide which segments live on the GPU.
//
// Restates the reference's CacheManager (src/gpudb/CacheManager.h:134-279,
// CacheManager.cu:34-97 pool and free list, :307-320 cacheSegmentInGPU,
// :534-588 SegmentReplacement, LRU/LFU replacement) for one device:
//   * one cudaMalloc'd pool of num_slots slots of segment_size ints (the kernels'
//     gpuCache), slot s at pool + s * segment_size;
//   * admission on demand (a query needs a segment that is not resident): take a free
//     slot, else evict the unpinned resident segment ranked lowest by the policy (LRU:
//     oldest use; LFU: fewest uses; WEIGHT: smallest planner-assigned benefit);
//   * epoch replacement (mb_segcache_replace): given a benefit weight per segment, keep
//     the highest-weighted positive segments that fit and evict the rest, as
//     SegmentReplacement does with the cost model's weights;
//   * a query stamp pins every segment the running query touched, so admission never
//     evicts a segment the same query still reads.
// Host-pool mode (device < 0) keeps the pool in host memory and copies with memcpy, so
// the bookkeeping runs without a GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "mordred_b200.h"

struct mb_segcache {
  int device;
  int64_t num_slots;
  int segment_size, num_columns, num_segments, policy;
  int* pool;
  std::vector<int> slot_of;        // [col * num_segments + seg] -> slot, -1 absent
  std::vector<int> owner;          // [slot] -> col * num_segments + seg, -1 free
  std::vector<uint64_t> last_use;  // per (col, seg)
  std::vector<uint64_t> uses;
  std::vector<double> weight;
  std::vector<int> free_slots;
  int64_t reserved = 0;            // the top `reserved` slots are the caller's (staging)
  uint64_t stamp = 1;
  mb_segcache_stats stats{};
  std::mutex mu;
};

namespace {

bool valid(const mb_segcache* c, int col, int seg) {
  return c && col >= 0 && col < c->num_columns && seg >= 0 && seg < c->num_segments;
}

int copy_in(mb_segcache* c, int slot, const int* src, int rows, cudaStream_t st) {
  int* dst = c->pool + static_cast<int64_t>(slot) * c->segment_size;
  const size_t bytes = static_cast<size_t>(rows) * 4;
  if (c->device < 0) {
    memcpy(dst, src, bytes);
    return MB_OK;
  }
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess ? MB_OK : MB_ERR_CUDA;
}

// Victim among resident, unpinned segments (lowest policy rank); -1 when none.
int pick_victim(const mb_segcache* c) {
  int best = -1;
  double best_key = 0;
  for (int64_t s = 0; s < c->num_slots; ++s) {
    const int k = c->owner[s];
    if (k < 0 || c->last_use[k] == c->stamp) continue;
    double key;
    if (c->policy == MB_CACHE_LFU)
      key = static_cast<double>(c->uses[k]);
    else if (c->policy == MB_CACHE_WEIGHT)
      key = c->weight[k];
    else
      key = static_cast<double>(c->last_use[k]);
    if (best < 0 || key < best_key) {
      best = static_cast<int>(s);
      best_key = key;
    }
  }
  return best;
}

void release(mb_segcache* c, int slot) {
  const int k = c->owner[slot];
  if (k < 0) return;
  c->slot_of[k] = -1;
  c->owner[slot] = -1;
  c->free_slots.push_back(slot);
  ++c->stats.evictions;
}

}  // namespace

extern "C" mb_segcache* mb_segcache_create(int device, int64_t num_slots, int segment_size, int num_columns,
                                           int num_segments, int policy) {
  if (num_slots <= 0 || segment_size <= 0 || (segment_size & (segment_size - 1)) != 0 || num_columns <= 0 ||
      num_segments <= 0 || num_segments > 32767 || policy < MB_CACHE_LRU || policy > MB_CACHE_WEIGHT)
    return nullptr;
  mb_segcache* c = new mb_segcache;
  c->device = device;
  c->num_slots = num_slots;
  c->segment_size = segment_size;
  c->num_columns = num_columns;
  c->num_segments = num_segments;
  c->policy = policy;
  const size_t bytes = static_cast<size_t>(num_slots) * segment_size * 4;
  if (device < 0) {
    c->pool = static_cast<int*>(aligned_alloc(256, (bytes + 255) / 256 * 256));
  } else {
    void* p = nullptr;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess || cudaMalloc(&p, bytes) != cudaSuccess) p = nullptr;
    cudaSetDevice(prev);
    c->pool = static_cast<int*>(p);
  }
  if (c->pool == nullptr) {
    delete c;
    return nullptr;
  }
  const size_t keys = static_cast<size_t>(num_columns) * num_segments;
  c->slot_of.assign(keys, -1);
  c->last_use.assign(keys, 0);
  c->uses.assign(keys, 0);
  c->weight.assign(keys, 0.0);
  c->owner.assign(num_slots, -1);
  for (int64_t s = num_slots - 1; s >= 0; --s) c->free_slots.push_back(static_cast<int>(s));
  return c;
}

extern "C" void mb_segcache_destroy(mb_segcache* c) {
  if (c == nullptr) return;
  if (c->device < 0)
    free(c->pool);
  else
    cudaFree(c->pool);
  delete c;
}

extern "C" int* mb_segcache_pool(mb_segcache* c) { return c ? c->pool : nullptr; }

extern "C" int mb_segcache_slot(mb_segcache* c, int col, int seg) {
  if (!valid(c, col, seg)) return -1;
  std::lock_guard<std::mutex> lk(c->mu);
  return c->slot_of[static_cast<size_t>(col) * c->num_segments + seg];
}

extern "C" int mb_segcache_col_idx(mb_segcache* c, int col, int* out) {
  if (c == nullptr || out == nullptr || col < 0 || col >= c->num_columns) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  memcpy(out, c->slot_of.data() + static_cast<size_t>(col) * c->num_segments, sizeof(int) * c->num_segments);
  return MB_OK;
}

extern "C" void mb_segcache_begin_query(mb_segcache* c) {
  if (c == nullptr) return;
  std::lock_guard<std::mutex> lk(c->mu);
  ++c->stamp;
}

extern "C" int mb_segcache_touch(mb_segcache* c, int col, int seg) {
  if (!valid(c, col, seg)) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  const size_t k = static_cast<size_t>(col) * c->num_segments + seg;
  c->last_use[k] = c->stamp;
  ++c->uses[k];
  if (c->slot_of[k] >= 0)
    ++c->stats.hits;
  else
    ++c->stats.misses;
  return MB_OK;
}

extern "C" int mb_segcache_set_weight(mb_segcache* c, int col, int seg, double w) {
  if (!valid(c, col, seg)) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  c->weight[static_cast<size_t>(col) * c->num_segments + seg] = w;
  return MB_OK;
}

extern "C" int mb_segcache_admit(mb_segcache* c, int col, int seg, const int* host_src, int rows,
                                 mb_stream_t stream, int* slot_out) {
  if (!valid(c, col, seg) || host_src == nullptr || rows < 0 || rows > c->segment_size) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  const size_t k = static_cast<size_t>(col) * c->num_segments + seg;
  c->last_use[k] = c->stamp;  // pinned for the running query
  if (c->slot_of[k] >= 0) {
    if (slot_out) *slot_out = c->slot_of[k];
    return MB_OK;
  }
  if (c->free_slots.empty()) {
    const int v = pick_victim(c);
    if (v < 0) return MB_ERR_SIZE;  // every slot holds a segment of the running query
    release(c, v);
  }
  const int slot = c->free_slots.back();
  const int e = copy_in(c, slot, host_src, rows, static_cast<cudaStream_t>(stream));
  if (e != MB_OK) return e;
  c->free_slots.pop_back();
  c->owner[slot] = static_cast<int>(k);
  c->slot_of[k] = slot;
  c->stats.bytes_h2d += static_cast<unsigned long long>(rows) * 4;
  ++c->stats.admissions;
  if (slot_out) *slot_out = slot;
  return MB_OK;
}

extern "C" int mb_segcache_admit_segments(mb_segcache* c, const int* cols, int ncols, const int* segs, int nsegs,
                                          const int* const* host_cols, const int* seg_rows, mb_stream_t stream,
                                          int* done, unsigned long long* copied) {
  if (c == nullptr || cols == nullptr || segs == nullptr || host_cols == nullptr || seg_rows == nullptr ||
      ncols < 0 || nsegs < 0 || done == nullptr)
    return MB_ERR_ARG;
  *done = 0;
  for (int i = 0; i < nsegs; ++i) {
    for (int j = 0; j < ncols; ++j) {
      const int col = cols[j], seg = segs[i];
      if (!valid(c, col, seg) || host_cols[col] == nullptr) return MB_ERR_ARG;
      {
        std::lock_guard<std::mutex> lk(c->mu);
        const size_t k = static_cast<size_t>(col) * c->num_segments + seg;
        ++c->uses[k];
        if (c->slot_of[k] >= 0)
          ++c->stats.hits;
        else
          ++c->stats.misses;
      }
      int slot = -1;
      const int had = mb_segcache_slot(c, col, seg);
      const int e = mb_segcache_admit(c, col, seg, host_cols[col] + static_cast<int64_t>(seg) * c->segment_size,
                                      seg_rows[seg], stream, &slot);
      if (e != MB_OK) return e;  // MB_ERR_SIZE: segment i does not fit beside the pinned ones
      if (had < 0 && copied) ++*copied;
    }
    *done = i + 1;
  }
  return MB_OK;
}

extern "C" int mb_segcache_evict(mb_segcache* c, int col, int seg) {
  if (!valid(c, col, seg)) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  const int s = c->slot_of[static_cast<size_t>(col) * c->num_segments + seg];
  if (s >= 0) release(c, s);
  return MB_OK;
}

extern "C" int mb_segcache_replace(mb_segcache* c, const double* weights, const int* const* host_cols,
                                   const int* segment_rows, mb_stream_t stream) {
  if (c == nullptr || weights == nullptr || host_cols == nullptr || segment_rows == nullptr) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  const size_t keys = static_cast<size_t>(c->num_columns) * c->num_segments;
  for (size_t k = 0; k < keys; ++k) c->weight[k] = weights[k];
  // the target set: positive weights, heaviest first, as many as there are slots
  std::vector<int> order;
  for (size_t k = 0; k < keys; ++k)
    if (weights[k] > 0) order.push_back(static_cast<int>(k));
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return weights[x] > weights[y]; });
  if (static_cast<int64_t>(order.size()) > c->num_slots - c->reserved) order.resize(c->num_slots - c->reserved);
  std::vector<char> keep(keys, 0);
  for (int k : order) keep[k] = 1;
  for (int64_t s = 0; s < c->num_slots; ++s)
    if (c->owner[s] >= 0 && !keep[c->owner[s]]) release(c, static_cast<int>(s));
  for (int k : order) {
    if (c->slot_of[k] >= 0) continue;
    const int col = k / c->num_segments, seg = k % c->num_segments;
    if (host_cols[col] == nullptr) continue;
    const int slot = c->free_slots.back();
    const int e = copy_in(c, slot, host_cols[col] + static_cast<int64_t>(seg) * c->segment_size, segment_rows[seg],
                          static_cast<cudaStream_t>(stream));
    if (e != MB_OK) return e;
    c->free_slots.pop_back();
    c->owner[slot] = k;
    c->slot_of[k] = slot;
    c->stats.bytes_h2d += static_cast<unsigned long long>(segment_rows[seg]) * 4;
    ++c->stats.admissions;
  }
  return MB_OK;
}

extern "C" int mb_segcache_get_stats(mb_segcache* c, mb_segcache_stats* out) {
  if (c == nullptr || out == nullptr) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  *out = c->stats;
  out->resident =
      static_cast<unsigned long long>(c->num_slots - c->reserved - static_cast<int64_t>(c->free_slots.size()));
  return MB_OK;
}

extern "C" int mb_segcache_reserve(mb_segcache* c, int64_t nslots, int64_t* first_slot) {
  if (c == nullptr || nslots < 0 || first_slot == nullptr) return MB_ERR_ARG;
  std::lock_guard<std::mutex> lk(c->mu);
  if (nslots >= c->num_slots - c->reserved) return MB_ERR_SIZE;
  const int64_t lo = c->num_slots - c->reserved - nslots, hi = c->num_slots - c->reserved;
  for (int64_t s = lo; s < hi; ++s)
    if (c->owner[s] >= 0) release(c, static_cast<int>(s));
  // take [lo, hi) out of the free list and out of every policy's reach
  std::vector<int> keep;
  keep.reserve(c->free_slots.size());
  for (int s : c->free_slots)
    if (s < lo || s >= hi) keep.push_back(s);
  c->free_slots.swap(keep);
  for (int64_t s = lo; s < hi; ++s) c->owner[s] = -2;
  c->reserved += nslots;
  *first_slot = lo;
  return MB_OK;
}

extern "C" int mb_segcache_stage(mb_segcache* c, int64_t slot, const int* host_src, int rows, mb_stream_t stream) {
  if (c == nullptr || host_src == nullptr || rows < 0 || rows > c->segment_size) return MB_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    if (slot < c->num_slots - c->reserved || slot >= c->num_slots) return MB_ERR_ARG;  // reserved slots only
    c->stats.bytes_h2d += static_cast<unsigned long long>(rows) * 4;
  }
  return copy_in(c, static_cast<int>(slot), host_src, rows, static_cast<cudaStream_t>(stream));
}
