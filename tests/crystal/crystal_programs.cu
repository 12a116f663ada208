// crystal_programs.cu — star-query programs written against the Crystal block-primitive API
// (include/crystal_b200.cuh), the way code written for Crystal uses it: one tile of
// BLOCK_THREADS x ITEMS_PER_THREAD fact rows per CTA, striped registers, int selection
// flags, perfect-hash builds and probes, BlockSum. Test infrastructure: they show that
// Crystal-style code compiles against the header and computes the oracle's answers.
//
// Query forms (constants are arguments): the filter-aggregate of src/ssb/q11.cu, the
// supplier -> part -> date probe of q21.cu grouped by (brand, year), and the
// supplier -> customer -> part -> date probe of q41.cu grouped by (c_nation, year).
#include <cuda_runtime.h>

#include "crystal_b200.cuh"

namespace {

constexpr int kThreads = 128;
constexpr int kItems = 4;
constexpr int kTile = kThreads * kItems;

__device__ __forceinline__ int tile_items(int n) {
  const int base = blockIdx.x * kTile;
  return n - base < kTile ? n - base : kTile;
}

__device__ __forceinline__ bool in_tile(int i, int items) { return static_cast<int>(threadIdx.x) + i * kThreads < items; }

template <int BT, int IPT>
__global__ void filter_aggregate(int* od, int* disc, int* qty, int* price, int n, int d_first, int d_last, int k_lo,
                                 int k_hi, int q_below, unsigned long long* revenue) {
  const int base = blockIdx.x * BT * IPT;
  const int items = tile_items(n);
  int v[IPT], w[IPT], sel[IPT];
  InitFlags<BT, IPT>(sel);
  BlockLoad<int, BT, IPT>(od + base, v, items);
  BlockPredAndGTE<int, BT, IPT>(v, d_first, sel, items);
  BlockPredAndLTE<int, BT, IPT>(v, d_last, sel, items);
  BlockLoad<int, BT, IPT>(qty + base, v, items);
  BlockPredAndLT<int, BT, IPT>(v, q_below, sel, items);
  BlockLoad<int, BT, IPT>(disc + base, v, items);
  BlockPredAndGTE<int, BT, IPT>(v, k_lo, sel, items);
  BlockPredAndLTE<int, BT, IPT>(v, k_hi, sel, items);
  BlockLoad<int, BT, IPT>(price + base, w, items);
  long long part = 0;
#pragma unroll
  for (int i = 0; i < IPT; ++i)
    if (in_tile(i, items) && sel[i]) part += static_cast<long long>(static_cast<int>(static_cast<unsigned>(w[i]) *
                                                                                        static_cast<unsigned>(v[i])));
  __shared__ long long scratch[32];
  const long long total = BlockSum<long long, BT, IPT>(part, scratch);
  if (threadIdx.x == 0 && total != 0) atomicAdd(revenue, static_cast<unsigned long long>(total));
}

// Filtered build of a PHT_1 (keys only) or PHT_2 ({key, value}) table: rows with
// filter == eq_a (or == eq_b when eq_b >= 0); no filter when filter is null.
template <int BT, int IPT>
__global__ void build_table(int* filter, int eq_a, int eq_b, int* key, int* val, int n, int* ht, int slots,
                            int keys_min) {
  const int base = blockIdx.x * BT * IPT;
  const int items = tile_items(n);
  int k[IPT], x[IPT], sel[IPT];
  InitFlags<BT, IPT>(sel);
  if (filter != nullptr) {
    BlockLoad<int, BT, IPT>(filter + base, x, items);
    BlockPredEQ<int, BT, IPT>(x, eq_a, sel, items);
    if (eq_b >= 0) BlockPredOrEQ<int, BT, IPT>(x, eq_b, sel, items);
  }
  BlockLoad<int, BT, IPT>(key + base, k, items);
  if (val == nullptr) {
    BlockBuildSelectivePHT_1<int, BT, IPT>(k, sel, ht, slots, keys_min, items);
  } else {
    BlockLoad<int, BT, IPT>(val + base, x, items);
    BlockBuildSelectivePHT_2<int, int, BT, IPT>(k, x, sel, ht, slots, keys_min, items);
  }
}

// supplier (existence) -> part (brand) -> date (year); group brand * 7 + year - 1992
template <int BT, int IPT>
__global__ void probe_brand_year(int* od, int* pk, int* sk, int* rev, int n, int* ht_s, int s_slots, int* ht_p,
                                 int p_slots, int* ht_d, int d_slots, int* res) {
  const int base = blockIdx.x * BT * IPT;
  const int items = tile_items(n);
  int k[IPT], sel[IPT], brand[IPT], year[IPT], r[IPT];
  InitFlags<BT, IPT>(sel);
  BlockLoad<int, BT, IPT>(sk + base, k, items);
  BlockProbeAndPHT_1<int, BT, IPT>(k, sel, ht_s, s_slots, items);
  BlockLoad<int, BT, IPT>(pk + base, k, items);
  BlockProbeAndPHT_2<int, int, BT, IPT>(k, brand, sel, ht_p, p_slots, items);
  BlockLoad<int, BT, IPT>(od + base, k, items);
  BlockProbeAndPHT_2<int, int, BT, IPT>(k, year, sel, ht_d, d_slots, 19920101, items);
  BlockLoad<int, BT, IPT>(rev + base, r, items);
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    if (!in_tile(i, items) || !sel[i]) continue;
    const int g = (brand[i] * 7 + year[i] - 1992) % 7000;
    res[4 * g] = year[i];
    res[4 * g + 1] = brand[i];
    atomicAdd(reinterpret_cast<unsigned long long*>(res + 4 * g + 2), static_cast<unsigned long long>(
                                                                            static_cast<long long>(r[i])));
  }
}

// supplier -> customer (nation) -> part -> date (year); group nation * 7 + year - 1992,
// summing revenue - supplycost (the difference in 32 bits)
template <int BT, int IPT>
__global__ void probe_nation_year(int* od, int* pk, int* ck, int* sk, int* rev, int* cost, int n, int* ht_p,
                                  int p_slots, int* ht_s, int s_slots, int* ht_c, int c_slots, int* ht_d, int d_slots,
                                  int* res) {
  const int base = blockIdx.x * BT * IPT;
  const int items = tile_items(n);
  int k[IPT], sel[IPT], nation[IPT], year[IPT], r[IPT];
  InitFlags<BT, IPT>(sel);
  BlockLoad<int, BT, IPT>(sk + base, k, items);
  BlockProbeAndPHT_1<int, BT, IPT>(k, sel, ht_s, s_slots, items);
  BlockLoad<int, BT, IPT>(ck + base, k, items);
  BlockProbeAndPHT_2<int, int, BT, IPT>(k, nation, sel, ht_c, c_slots, items);
  BlockLoad<int, BT, IPT>(pk + base, k, items);
  BlockProbeAndPHT_1<int, BT, IPT>(k, sel, ht_p, p_slots, items);
  BlockLoad<int, BT, IPT>(od + base, k, items);
  BlockProbeAndPHT_2<int, int, BT, IPT>(k, year, sel, ht_d, d_slots, 19920101, items);
  BlockLoad<int, BT, IPT>(rev + base, r, items);
  BlockLoad<int, BT, IPT>(cost + base, k, items);
#pragma unroll
  for (int i = 0; i < IPT; ++i) {
    if (!in_tile(i, items) || !sel[i]) continue;
    const int g = (nation[i] * 7 + year[i] - 1992) % 175;
    res[4 * g] = year[i];
    res[4 * g + 1] = nation[i];
    const int profit = static_cast<int>(static_cast<unsigned>(r[i]) - static_cast<unsigned>(k[i]));
    atomicAdd(reinterpret_cast<unsigned long long*>(res + 4 * g + 2),
              static_cast<unsigned long long>(static_cast<long long>(profit)));
  }
}

int grid(int n) { return n > 0 ? (n + kTile - 1) / kTile : 0; }

int finish() {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return static_cast<int>(e);
}

}  // namespace

extern "C" {

int cp_filter_aggregate(int* od, int* disc, int* qty, int* price, int n, unsigned long long* revenue) {
  if (n <= 0) return 0;
  filter_aggregate<kThreads, kItems><<<grid(n), kThreads>>>(od, disc, qty, price, n, 19930101, 19931231, 1, 3, 25,
                                                             revenue);
  return finish();
}

int cp_build(int* filter, int eq_a, int eq_b, int* key, int* val, int n, int* ht, int slots, int keys_min) {
  if (n <= 0) return 0;
  build_table<kThreads, kItems><<<grid(n), kThreads>>>(filter, eq_a, eq_b, key, val, n, ht, slots, keys_min);
  return finish();
}

int cp_probe_brand_year(int* od, int* pk, int* sk, int* rev, int n, int* ht_s, int s_slots, int* ht_p, int p_slots,
                        int* ht_d, int d_slots, int* res) {
  if (n <= 0) return 0;
  probe_brand_year<kThreads, kItems><<<grid(n), kThreads>>>(od, pk, sk, rev, n, ht_s, s_slots, ht_p, p_slots, ht_d,
                                                             d_slots, res);
  return finish();
}

int cp_probe_nation_year(int* od, int* pk, int* ck, int* sk, int* rev, int* cost, int n, int* ht_p, int p_slots,
                         int* ht_s, int s_slots, int* ht_c, int c_slots, int* ht_d, int d_slots, int* res) {
  if (n <= 0) return 0;
  probe_nation_year<kThreads, kItems><<<grid(n), kThreads>>>(od, pk, ck, sk, rev, cost, n, ht_p, p_slots, ht_s,
                                                              s_slots, ht_c, c_slots, ht_d, d_slots, res);
  return finish();
}

}  // extern "C"
