/*
 * crystal_b200.cuh — the Crystal block-wide primitive API for sm_100a.
 *
 * Code written against Crystal (the reference's crystal/crystal.cuh: load.cuh, pred.cuh,
 * store.cuh, reduce.cuh, join.cuh) compiles against this header unchanged: the template
 * names, template parameter lists and argument lists below are Crystal's, and so are the
 * data conventions the callers rely on —
 *   - a tile of BLOCK_THREADS * ITEMS_PER_THREAD items is held striped: thread t holds
 *     items t, t + BLOCK_THREADS, t + 2 * BLOCK_THREADS, ... (crystal/load.cuh:9-14);
 *   - selection flags are one int per item (1 selected, 0 not);
 *   - perfect hash: slot = (key - keys_min) % ht_len (crystal/join.cuh:3); PHT_1 tables
 *     hold the key in slot s (0 = empty); PHT_2 tables hold {key, value} pairs and a probe
 *     reads the 8-byte pair, nonzero = present, value = its upper 32 bits
 *     (crystal/join.cuh:84-165, 236-311);
 *   - BlockSum leaves the block total in thread 0 (crystal/reduce.cuh:4-53).
 *
 * What is B200-specific is inside: fact-column loads are streaming loads (ld.global.cs:
 * evict-first, so a scan does not push the probed hash tables out of L2); hash-table
 * reads go through the read-only path (ld.global.nc) as one 8-byte load per PHT_2 slot;
 * the slot of a key in [keys_min, keys_min + 2 * ht_len) is found without a division
 * (the same value the remainder gives); 32-bit block sums reduce each warp with the
 * hardware warp reduction (redux.sync) and wider types with register shuffles.
 *
 * One deliberate difference: a key whose slot comes out negative (a key below keys_min)
 * reads or writes before the table in the reference; here a probe drops such an item and
 * a build skips it.
 *
 * Header-only; include it where the reference includes "crystal/crystal.cuh".
 */
#ifndef CRYSTAL_B200_CUH
#define CRYSTAL_B200_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef HASH
#define HASH(X, Y, Z) ((X - Z) % Y)
#endif

namespace crystal_b200 {

/* Streaming load of a scanned column item (evict-first in L1 and L2). */
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) { return *p; }
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }
__device__ __forceinline__ unsigned ld_stream(const unsigned* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ long long ld_stream(const long long* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }

/* Read-only load of a hash-table word. */
template <typename T>
__device__ __forceinline__ T ld_table(const T* p) { return *p; }
__device__ __forceinline__ int ld_table(const int* p) { return __ldg(p); }
__device__ __forceinline__ unsigned ld_table(const unsigned* p) { return __ldg(p); }
__device__ __forceinline__ long long ld_table(const long long* p) { return __ldg(p); }
__device__ __forceinline__ unsigned long long ld_table(const unsigned long long* p) { return __ldg(p); }

/* (key - keys_min) % ht_len in the key type's arithmetic, without the division for keys in
 * [keys_min, keys_min + 2 * ht_len). Returns a negative value for keys below keys_min. */
template <typename K>
__device__ __forceinline__ int slot(K key, int ht_len, K keys_min) {
  const K d = key - keys_min;
  if (d >= 0 && d < static_cast<K>(ht_len)) return static_cast<int>(d);
  if (d >= static_cast<K>(ht_len) && d < static_cast<K>(2) * static_cast<K>(ht_len) && ht_len <= (1 << 30))
    return static_cast<int>(d - static_cast<K>(ht_len));
  return static_cast<int>(d % ht_len);
}
template <>
__device__ __forceinline__ int slot<int>(int key, int ht_len, int keys_min) {
  const int d = static_cast<int>(static_cast<unsigned>(key) - static_cast<unsigned>(keys_min));
  if (static_cast<unsigned>(d) < static_cast<unsigned>(ht_len)) return d;
  if (static_cast<unsigned>(d) < 2u * static_cast<unsigned>(ht_len) && ht_len <= (1 << 30)) return d - ht_len;
  return d % ht_len;
}

/* Sum over a warp: the hardware reduction for 32-bit integers, shuffles otherwise. The
 * result is valid in lane 0 (in every lane for the 32-bit forms). */
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum(int v) { return __reduce_add_sync(0xffffffffu, v); }
__device__ __forceinline__ unsigned warp_sum(unsigned v) { return __reduce_add_sync(0xffffffffu, v); }

}  // namespace crystal_b200

/* ---- load (crystal/load.cuh) ------------------------------------------------------- */

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoadDirect(const unsigned int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD]) {
  const T* p = block_itr + tid;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS);
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoadDirect(const unsigned int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD],
                                                int num_items) {
  const T* p = block_itr + tid;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i)
    if (static_cast<int>(tid) + i * BLOCK_THREADS < num_items) items[i] = crystal_b200::ld_stream(p + i * BLOCK_THREADS);
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoad(T* inp, T (&items)[ITEMS_PER_THREAD], int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockLoadDirect<T, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, inp, items);
  else
    BlockLoadDirect<T, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, inp, items, num_items);
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockLoadCrystal(T* inp, T (&items)[ITEMS_PER_THREAD], int num_items) {
  BlockLoad<T, BLOCK_THREADS, ITEMS_PER_THREAD>(inp, items, num_items);
}

/* ---- store (crystal/store.cuh) ----------------------------------------------------- */

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockStoreDirect(int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD]) {
  T* p = block_itr + tid;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) p[i * BLOCK_THREADS] = items[i];
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockStoreDirect(int tid, T* block_itr, T (&items)[ITEMS_PER_THREAD], int num_items) {
  T* p = block_itr + tid;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i)
    if (tid + i * BLOCK_THREADS < num_items) p[i * BLOCK_THREADS] = items[i];
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockStore(T* out, T (&items)[ITEMS_PER_THREAD], int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockStoreDirect<T, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, out, items);
  else
    BlockStoreDirect<T, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, out, items, num_items);
}

/* ---- predicates (crystal/pred.cuh) ------------------------------------------------- */

template <int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void InitFlags(int (&selection_flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) selection_flags[i] = 1;
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredDirect(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                                int (&selection_flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) selection_flags[i] = select_op(items[i]);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredDirect(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                                int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i)
    if (tid + i * BLOCK_THREADS < num_items) selection_flags[i] = select_op(items[i]);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPred(T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                          int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockPredDirect<T, SelectOp, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, select_op, selection_flags);
  else
    BlockPredDirect<T, SelectOp, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, select_op, selection_flags,
                                                                   num_items);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredAndDirect(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                                   int (&selection_flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) selection_flags[i] = selection_flags[i] && select_op(items[i]);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredAndDirect(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                                   int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i)
    if (tid + i * BLOCK_THREADS < num_items) selection_flags[i] = selection_flags[i] && select_op(items[i]);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredAnd(T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                             int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockPredAndDirect<T, SelectOp, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, select_op, selection_flags);
  else
    BlockPredAndDirect<T, SelectOp, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, select_op, selection_flags,
                                                                      num_items);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredOrDirect(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                                  int (&selection_flags)[ITEMS_PER_THREAD]) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) selection_flags[i] = selection_flags[i] || select_op(items[i]);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredOrDirect(int tid, T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                                  int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i)
    if (tid + i * BLOCK_THREADS < num_items) selection_flags[i] = selection_flags[i] || select_op(items[i]);
}

template <typename T, typename SelectOp, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockPredOr(T (&items)[ITEMS_PER_THREAD], SelectOp select_op,
                                            int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockPredOrDirect<T, SelectOp, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, select_op, selection_flags);
  else
    BlockPredOrDirect<T, SelectOp, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, select_op, selection_flags,
                                                                     num_items);
}

/* Comparison functors: a single member `compare`, constructed from it. */
template <typename T>
struct LessThan {
  T compare;
  __device__ __forceinline__ LessThan(T c) : compare(c) {}
  __device__ __forceinline__ bool operator()(const T& a) const { return a < compare; }
};
template <typename T>
struct GreaterThan {
  T compare;
  __device__ __forceinline__ GreaterThan(T c) : compare(c) {}
  __device__ __forceinline__ bool operator()(const T& a) const { return a > compare; }
};
template <typename T>
struct LessThanEq {
  T compare;
  __device__ __forceinline__ LessThanEq(T c) : compare(c) {}
  __device__ __forceinline__ bool operator()(const T& a) const { return a <= compare; }
};
template <typename T>
struct GreaterThanEq {
  T compare;
  __device__ __forceinline__ GreaterThanEq(T c) : compare(c) {}
  __device__ __forceinline__ bool operator()(const T& a) const { return a >= compare; }
};
template <typename T>
struct Eq {
  T compare;
  __device__ __forceinline__ Eq(T c) : compare(c) {}
  __device__ __forceinline__ bool operator()(const T& a) const { return a == compare; }
};

#define CRYSTAL_B200_PRED(NAME, COMBINE, OP)                                                                   \
  template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>                                                \
  __device__ __forceinline__ void NAME(T (&items)[ITEMS_PER_THREAD], T compare,                                 \
                                       int (&selection_flags)[ITEMS_PER_THREAD], int num_items) {               \
    COMBINE<T, OP<T>, BLOCK_THREADS, ITEMS_PER_THREAD>(items, OP<T>(compare), selection_flags, num_items);      \
  }
CRYSTAL_B200_PRED(BlockPredLT, BlockPred, LessThan)
CRYSTAL_B200_PRED(BlockPredAndLT, BlockPredAnd, LessThan)
CRYSTAL_B200_PRED(BlockPredGT, BlockPred, GreaterThan)
CRYSTAL_B200_PRED(BlockPredAndGT, BlockPredAnd, GreaterThan)
CRYSTAL_B200_PRED(BlockPredLTE, BlockPred, LessThanEq)
CRYSTAL_B200_PRED(BlockPredAndLTE, BlockPredAnd, LessThanEq)
CRYSTAL_B200_PRED(BlockPredGTE, BlockPred, GreaterThanEq)
CRYSTAL_B200_PRED(BlockPredAndGTE, BlockPredAnd, GreaterThanEq)
CRYSTAL_B200_PRED(BlockPredEQ, BlockPred, Eq)
CRYSTAL_B200_PRED(BlockPredAndEQ, BlockPredAnd, Eq)
CRYSTAL_B200_PRED(BlockPredOrEQ, BlockPredOr, Eq)
#undef CRYSTAL_B200_PRED

/* ---- block sum (crystal/reduce.cuh) ------------------------------------------------ */

/* Sum of `item` over the block, valid in thread 0. `shared` holds at least one T per warp. */
template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ T BlockSum(T item, T* shared) {
  __syncthreads();  // earlier users of `shared` are done
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T v = crystal_b200::warp_sum(item);
  if (lane == 0) shared[wid] = v;
  __syncthreads();
  v = threadIdx.x < blockDim.x / 32 ? shared[lane] : T(0);
  if (wid == 0) v = crystal_b200::warp_sum(v);
  return v;
}

template <typename T, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ T BlockSum(T (&items)[ITEMS_PER_THREAD], T* shared) {
  T s = 0;
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) s += items[i];
  return BlockSum<T, BLOCK_THREADS, ITEMS_PER_THREAD>(s, shared);
}

/* ---- perfect-hash probe and build (crystal/join.cuh) ------------------------------- */

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (!selection_flags[i]) continue;
    const int h = crystal_b200::slot(items[i], ht_len, keys_min);
    selection_flags[i] = h >= 0 && crystal_b200::ld_table(ht + h) != K(0);
  }
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_1(int tid, K (&items)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (tid + i * BLOCK_THREADS >= num_items || !selection_flags[i]) continue;
    const int h = crystal_b200::slot(items[i], ht_len, keys_min);
    selection_flags[i] = h >= 0 && crystal_b200::ld_table(ht + h) != K(0);
  }
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_1(K (&items)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   K keys_min, int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockProbeDirectAndPHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, selection_flags, ht, ht_len,
                                                                  keys_min);
  else
    BlockProbeDirectAndPHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, items, selection_flags, ht, ht_len,
                                                                  keys_min, num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_1(K (&items)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   int num_items) {
  BlockProbeAndPHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(items, selection_flags, ht, ht_len, K(0), num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_2(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                         V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (!selection_flags[i]) continue;
    const int h = crystal_b200::slot(keys[i], ht_len, keys_min);
    const unsigned long long s =
        h >= 0 ? crystal_b200::ld_table(reinterpret_cast<const unsigned long long*>(ht + 2ll * h)) : 0ull;
    if (s != 0ull)
      res[i] = static_cast<V>(s >> 32);
    else
      selection_flags[i] = 0;
  }
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeDirectAndPHT_2(int tid, K (&items)[ITEMS_PER_THREAD],
                                                         V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (tid + i * BLOCK_THREADS >= num_items || !selection_flags[i]) continue;
    const int h = crystal_b200::slot(items[i], ht_len, keys_min);
    const unsigned long long s =
        h >= 0 ? crystal_b200::ld_table(reinterpret_cast<const unsigned long long*>(ht + 2ll * h)) : 0ull;
    if (s != 0ull)
      res[i] = static_cast<V>(s >> 32);
    else
      selection_flags[i] = 0;
  }
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   K keys_min, int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockProbeDirectAndPHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, keys, res, selection_flags, ht,
                                                                     ht_len, keys_min);
  else
    BlockProbeDirectAndPHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, keys, res, selection_flags, ht,
                                                                     ht_len, keys_min, num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockProbeAndPHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                   int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                   int num_items) {
  BlockProbeAndPHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, K(0), num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_1(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (!selection_flags[i]) continue;
    const int h = crystal_b200::slot(keys[i], ht_len, keys_min);
    if (h >= 0) atomicCAS(ht + h, K(0), keys[i]);
  }
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_1(int tid, K (&items)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min, int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (tid + i * BLOCK_THREADS >= num_items || !selection_flags[i]) continue;
    const int h = crystal_b200::slot(items[i], ht_len, keys_min);
    if (h >= 0) atomicCAS(ht + h, K(0), items[i]);
  }
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_1(K (&keys)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockBuildDirectSelectivePHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, keys, selection_flags, ht, ht_len,
                                                                        keys_min);
  else
    BlockBuildDirectSelectivePHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, keys, selection_flags, ht, ht_len,
                                                                        keys_min, num_items);
}

template <typename K, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_1(K (&keys)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         int num_items) {
  BlockBuildSelectivePHT_1<K, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, selection_flags, ht, ht_len, K(0), num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                               V (&res)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (!selection_flags[i]) continue;
    const int h = crystal_b200::slot(keys[i], ht_len, keys_min);
    if (h < 0) continue;
    atomicCAS(ht + 2ll * h, K(0), keys[i]);
    ht[2ll * h + 1] = res[i];
  }
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildDirectSelectivePHT_2(int tid, K (&keys)[ITEMS_PER_THREAD],
                                                               V (&res)[ITEMS_PER_THREAD],
                                                               int (&selection_flags)[ITEMS_PER_THREAD], K* ht,
                                                               int ht_len, K keys_min, int num_items) {
#pragma unroll
  for (int i = 0; i < ITEMS_PER_THREAD; ++i) {
    if (tid + i * BLOCK_THREADS >= num_items || !selection_flags[i]) continue;
    const int h = crystal_b200::slot(keys[i], ht_len, keys_min);
    if (h < 0) continue;
    atomicCAS(ht + 2ll * h, K(0), keys[i]);
    ht[2ll * h + 1] = res[i];
  }
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         K keys_min, int num_items) {
  if (BLOCK_THREADS * ITEMS_PER_THREAD == num_items)
    BlockBuildDirectSelectivePHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, keys, res, selection_flags, ht,
                                                                           ht_len, keys_min);
  else
    BlockBuildDirectSelectivePHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(threadIdx.x, keys, res, selection_flags, ht,
                                                                           ht_len, keys_min, num_items);
}

template <typename K, typename V, int BLOCK_THREADS, int ITEMS_PER_THREAD>
__device__ __forceinline__ void BlockBuildSelectivePHT_2(K (&keys)[ITEMS_PER_THREAD], V (&res)[ITEMS_PER_THREAD],
                                                         int (&selection_flags)[ITEMS_PER_THREAD], K* ht, int ht_len,
                                                         int num_items) {
  BlockBuildSelectivePHT_2<K, V, BLOCK_THREADS, ITEMS_PER_THREAD>(keys, res, selection_flags, ht, ht_len, K(0),
                                                                  num_items);
}

#endif /* CRYSTAL_B200_CUH */
