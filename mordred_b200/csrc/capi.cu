// capi.cu — extern "C" entry points: runtime state, the generic fused star query, the
// SSB-signature wrappers, the engine (src/gpudb) wrappers and the synthetic generator.
#include <atomic>
#include <climits>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "ssbgen.h"
#include "star.cuh"

namespace mb {

static std::mutex g_state_mu;
static DeviceState g_state[64];
static std::atomic<unsigned long long> g_launches{0};

void note_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static int init_device_locked(int dev) {
  DeviceState& ds = g_state[dev];
  if (ds.device == dev) return MB_OK;
  int sms = 0, optin = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MB_ERR_NODEV;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return MB_ERR_NODEV;
  unsigned int* status = nullptr;
  if (cudaMalloc(&status, sizeof(unsigned int)) != cudaSuccess) return MB_ERR_CUDA;
  if (cudaMemset(status, 0, sizeof(unsigned int)) != cudaSuccess) return MB_ERR_CUDA;
  ds.num_sms = sms;
  ds.max_smem_optin = optin;
  ds.status = status;
  int e = star_init_device(ds);
  if (e == MB_OK) e = batch_init_device(ds);
  if (e == MB_OK) e = list_init_device(ds);
  if (e != MB_OK) return e;
  ds.device = dev;
  return MB_OK;
}

DeviceState* current_device_state(int* err) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    *err = MB_ERR_NODEV;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_state_mu);
  int e = init_device_locked(dev);
  if (e != MB_OK) {
    *err = e;
    return nullptr;
  }
  return &g_state[dev];
}

// ---- generator kernels ---------------------------------------------------------------
__global__ void gen_fact_kernel(int col, uint64_t seed, long long row0, long long n, int s_len, int c_len,
                                int p_len, int* out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    out[i] = mb_gen_fact_value(seed, col, static_cast<uint64_t>(row0 + i), s_len, c_len, p_len);
}

__global__ void gen_dim_kernel(int col, uint64_t seed, long long n, int* out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    out[i] = mb_gen_dim_value(seed, col, static_cast<uint64_t>(i));
}

template <class F>
static void host_parallel(long long n, int nthreads, F&& f) {
  if (nthreads <= 0) nthreads = static_cast<int>(std::thread::hardware_concurrency());
  if (nthreads < 1) nthreads = 1;
  if (n < 65536) nthreads = 1;
  std::vector<std::thread> ts;
  const long long chunk = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    const long long lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
    if (lo >= hi) break;
    ts.emplace_back([=, &f] { f(lo, hi); });
  }
  for (auto& t : ts) t.join();
}

}  // namespace mb

using namespace mb;

extern "C" {

int mb_version(void) { return 1; }

int mb_init(int device) {
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) return MB_ERR_NODEV;
  if (device < 0) device = cur;
  if (device >= 64) return MB_ERR_ARG;
  if (device != cur && cudaSetDevice(device) != cudaSuccess) return MB_ERR_NODEV;
  int e;
  {
    std::lock_guard<std::mutex> lk(g_state_mu);
    e = init_device_locked(device);
  }
  if (device != cur) cudaSetDevice(cur);
  return e;
}

int mb_device_status(int device, unsigned int* status, int clear) {
  if (status == nullptr) return MB_ERR_ARG;
  int e = mb_init(device);
  if (e != MB_OK) return e;
  int cur = -1;
  cudaGetDevice(&cur);
  if (device < 0) device = cur;
  if (device != cur) cudaSetDevice(device);
  unsigned int* d = g_state[device].status;
  e = MB_OK;
  if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(status, d, sizeof(unsigned int), cudaMemcpyDeviceToHost) != cudaSuccess)
    e = MB_ERR_CUDA;
  if (e == MB_OK && clear && cudaMemset(d, 0, sizeof(unsigned int)) != cudaSuccess) e = MB_ERR_CUDA;
  if (device != cur) cudaSetDevice(cur);
  return e;
}

const char* mb_error_string(int code) {
  switch (code) {
    case MB_OK: return "ok";
    case MB_ERR_ARG: return "invalid argument";
    case MB_ERR_ALIGN: return "misaligned pointer";
    case MB_ERR_LAUNCH: return "kernel launch failed";
    case MB_ERR_CUDA: return "CUDA runtime error";
    case MB_ERR_NODEV: return "no usable CUDA device";
    case MB_ERR_SIZE: return "size beyond the supported maximum";
    default: return "unknown error";
  }
}

unsigned long long mb_launch_count(void) { return g_launches.load(); }

int mb_device_state_ready(int device) {
  if (device < 0 || device >= 64) return 0;
  std::lock_guard<std::mutex> lk(g_state_mu);
  return g_state[device].device == device ? 1 : 0;
}

int mb_star_query(const mb_star_args* args, mb_stream_t stream) {
  return launch_star(args, static_cast<cudaStream_t>(stream), 0);
}

// ---- SSB signatures ------------------------------------------------------------------
int mb_q11_query(const int* lo_orderdate, const int* lo_discount, const int* lo_quantity,
                 const int* lo_extendedprice, int lo_num_entries, unsigned long long* revenue, int* d_total,
                 mb_stream_t stream) {
  if (lo_num_entries == 0) return MB_OK;
  if (!lo_orderdate || !lo_discount || !lo_quantity || !lo_extendedprice || !revenue || lo_num_entries < 0)
    return MB_ERR_ARG;
  mb_star_args a;
  memset(&a, 0, sizeof(a));
  a.num_rows = lo_num_entries;
  a.num_filters = 3;
  // q11.cu:46-64: discount in [1,3], quantity < 25, 19930000 < orderdate < 19940000
  a.filter[0] = {lo_discount, MB_FILTER_BETWEEN, 1, 3};
  a.filter[1] = {lo_quantity, MB_FILTER_BETWEEN, INT_MIN, 24};
  a.filter[2] = {lo_orderdate, MB_FILTER_BETWEEN, 19930001, 19939999};
  a.aggr[0] = lo_extendedprice;
  a.aggr[1] = lo_discount;
  a.agg_op = MB_AGG_MUL;
  a.total_val = 1;
  a.res_layout = MB_RES_SCALAR;
  a.res = revenue;
  a.count = reinterpret_cast<unsigned long long*>(d_total);
  a.count_after = 2;  // d_total counts rows passing the discount and quantity predicates (q11.cu:53-60)
  return launch_star(&a, static_cast<cudaStream_t>(stream), 1);
}

int mb_q21_probe(const int* lo_orderdate, const int* lo_partkey, const int* lo_suppkey, const int* lo_revenue,
                 int lo_len, const int* ht_s, int s_len, const int* ht_p, int p_len, const int* ht_d, int d_len,
                 int* res, mb_stream_t stream) {
  mb_star_args a;
  memset(&a, 0, sizeof(a));
  a.num_rows = lo_len;
  a.num_probes = 3;
  // q21.cu:48-57: supplier existence, part -> brand, date -> year (keys_min 19920101)
  a.probe[0] = {lo_suppkey, ht_s, s_len, 0, MB_HT_KEY, 0, 0, -1, nullptr};
  a.probe[1] = {lo_partkey, ht_p, p_len, 0, MB_HT_KEY_VAL, 0, 7, 1, nullptr};
  a.probe[2] = {lo_orderdate, ht_d, d_len, 19920101, MB_HT_KEY_VAL, 1992, 1, 0, nullptr};
  a.aggr[0] = lo_revenue;
  a.agg_op = MB_AGG_SUM;
  a.total_val = (1998 - 1992 + 1) * (5 * 5 * 40);  // q21.cu:65
  a.res_layout = MB_RES_CRYSTAL4;
  a.res = res;
  a.count_after = -1;
  return launch_star(&a, static_cast<cudaStream_t>(stream), 0);
}

int mb_q41_probe(const int* lo_orderdate, const int* lo_partkey, const int* lo_custkey, const int* lo_suppkey,
                 const int* lo_revenue, const int* lo_supplycost, int lo_len, const int* ht_p, int p_len,
                 const int* ht_s, int s_len, const int* ht_c, int c_len, const int* ht_d, int d_len, int* res,
                 mb_stream_t stream) {
  mb_star_args a;
  memset(&a, 0, sizeof(a));
  a.num_rows = lo_len;
  a.num_probes = 4;
  // q41.cu:50-62: supplier, customer -> nation, part, date -> year
  a.probe[0] = {lo_suppkey, ht_s, s_len, 0, MB_HT_KEY, 0, 0, -1, nullptr};
  a.probe[1] = {lo_custkey, ht_c, c_len, 0, MB_HT_KEY_VAL, 0, 7, 1, nullptr};
  a.probe[2] = {lo_partkey, ht_p, p_len, 0, MB_HT_KEY, 0, 0, -1, nullptr};
  a.probe[3] = {lo_orderdate, ht_d, d_len, 19920101, MB_HT_KEY_VAL, 1992, 1, 0, nullptr};
  a.aggr[0] = lo_revenue;
  a.aggr[1] = lo_supplycost;
  a.agg_op = MB_AGG_SUB;
  a.total_val = (1998 - 1992 + 1) * 25;  // q41.cu:71
  a.res_layout = MB_RES_CRYSTAL4;
  a.res = res;
  a.count_after = -1;
  return launch_star(&a, static_cast<cudaStream_t>(stream), 0);
}

int mb_join_probe(const int* fact_fkey, const int* fact_val, int num_tuples, const int* hash_table, int num_slots,
                  unsigned long long* res, mb_stream_t stream) {
  // src/ops/join.cu:62-73: PHT_2 probe, sum of fact_val * dim_val (int32 product)
  if (num_tuples == 0) return MB_OK;
  if (!fact_fkey || !fact_val || !hash_table || !res) return MB_ERR_ARG;
  mb_star_args a;
  memset(&a, 0, sizeof(a));
  a.num_rows = num_tuples;
  a.num_probes = 1;
  a.probe[0] = {fact_fkey, hash_table, num_slots, 0, MB_HT_KEY_VAL, 0, 0, -1, nullptr};
  a.aggr[0] = fact_val;
  a.agg_op = MB_AGG_MUL_PAYLOAD;
  a.total_val = 1;
  a.res_layout = MB_RES_SCALAR;
  a.res = res;
  a.count_after = -1;
  return launch_star(&a, static_cast<cudaStream_t>(stream), 0);
}

// ---- engine wrappers ---------------------------------------------------------------------
// Engine kernels restated on the fused pipeline. `off` (list forms) names the physical fact
// rows to visit and the dimension offsets earlier joins produced; slots whose group value
// comes from such an offset read gargs' dimension column there (MB_HT_PASS).
enum EngineFilters { kEngineBothFilters, kEngineSecondFilter };

static int engine_star(const int* gpuCache, const mb_offsetGPU* off, const mb_filterArgsGPU* fargs,
                       const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs, int num_tuples, int* res,
                       int start_offset, const short* segment_group, mb_stream_t stream, bool group_by,
                       bool probe_only_date, EngineFilters filters = kEngineBothFilters) {
  if (gargs == nullptr || res == nullptr || num_tuples < 0) return MB_ERR_ARG;
  if (off != nullptr && off->lo_off == nullptr) return MB_ERR_ARG;
  if (num_tuples == 0) return MB_OK;
  mb_star_args a;
  memset(&a, 0, sizeof(a));
  a.num_rows = num_tuples;
  a.rows = off != nullptr ? off->lo_off : nullptr;
  if (fargs != nullptr) {
    // fact-side filters are BETWEEN compare1..compare2 / compare3..compare4 (GPUProcessing.h:74-86);
    // filter_probe_aggr_GPU3 applies the second only (GPUProcessing.h:1808-1812)
    if (fargs->filter_idx1 && filters == kEngineBothFilters)
      a.filter[a.num_filters++] = {fargs->filter_idx1, MB_FILTER_BETWEEN, fargs->compare1, fargs->compare2};
    if (fargs->filter_idx2) a.filter[a.num_filters++] = {fargs->filter_idx2, MB_FILTER_BETWEEN, fargs->compare3, fargs->compare4};
  }
  static const mb_probeArgsGPU kNoProbes = {};
  if (pargs == nullptr) pargs = &kNoProbes;
  const int* keys[4] = {pargs->key_idx1, pargs->key_idx2, pargs->key_idx3, pargs->key_idx4};
  const int* hts[4] = {pargs->ht1, pargs->ht2, pargs->ht3, pargs->ht4};
  const int lens[4] = {pargs->dim_len1, pargs->dim_len2, pargs->dim_len3, pargs->dim_len4};
  const int kmins[4] = {pargs->min_key1, pargs->min_key2, pargs->min_key3, pargs->min_key4};
  const int mins[4] = {gargs->min_val1, gargs->min_val2, gargs->min_val3, gargs->min_val4};
  const int uniq[4] = {gargs->unique_val1, gargs->unique_val2, gargs->unique_val3, gargs->unique_val4};
  const int* groups[4] = {gargs->group_idx1, gargs->group_idx2, gargs->group_idx3, gargs->group_idx4};
  const int* doffs[4] = {off ? off->dim_off1 : nullptr, off ? off->dim_off2 : nullptr, off ? off->dim_off3 : nullptr,
                         off ? off->dim_off4 : nullptr};
  int bias = 0;
  for (int s = 0; s < 4; ++s) {
    if (probe_only_date && s != 3) continue;  // the aggregate kernels probe slot 4 only (GPUProcessing.h:1737)
    if (keys[s] != nullptr && hts[s] != nullptr) {
      a.probe[a.num_probes++] = {keys[s], hts[s], lens[s], kmins[s], MB_HT_VAL_OFF,
                                 mins[s], group_by ? uniq[s] : 0, group_by ? s : -1, nullptr};
    } else if (group_by && off != nullptr && groups[s] != nullptr) {
      // the value an earlier join found: the dimension column at the listed dimension row
      // (GPUProcessing.h:198-205); the reference does not bound the row, so neither is it
      // bounded here beyond being non-negative
      if (doffs[s] == nullptr) return MB_ERR_ARG;
      a.probe[a.num_probes++] = {doffs[s], groups[s], INT_MAX, 0, MB_HT_PASS, mins[s], uniq[s], s, nullptr};
    } else if (group_by) {
      // an absent probe contributes group value 0 (BlockSetValue, GPUProcessing.h:94-96)
      bias += static_cast<int>(static_cast<unsigned>(0 - mins[s]) * static_cast<unsigned>(uniq[s]));
    }
  }
  a.group_bias = bias;
  if (group_by) {
    // aggr1 - aggr2 with a missing column read as 0 (GPUProcessing.h:124-136,149)
    if (gargs->aggr_idx1 == nullptr && gargs->aggr_idx2 == nullptr) return MB_ERR_ARG;
    if (gargs->mode == 1) {
      if (!gargs->aggr_idx1 || !gargs->aggr_idx2) return MB_ERR_ARG;
      a.aggr[0] = gargs->aggr_idx1; a.aggr[1] = gargs->aggr_idx2; a.agg_op = MB_AGG_MUL;
    } else if (gargs->aggr_idx1 && gargs->aggr_idx2) {
      a.aggr[0] = gargs->aggr_idx1; a.aggr[1] = gargs->aggr_idx2; a.agg_op = MB_AGG_SUB;
    } else if (gargs->aggr_idx1) {
      a.aggr[0] = gargs->aggr_idx1; a.agg_op = MB_AGG_SUM;
    } else {
      return MB_ERR_ARG;  // 0 - aggr2 alone is not produced by the engine's planner
    }
    if (gargs->total_val <= 0) return MB_ERR_ARG;
    a.total_val = gargs->total_val;
    a.res_layout = MB_RES_ENGINE6;
    a.res = res;
  } else {
    // aggr1 * aggr2 summed into the u64 at res[4] (GPUProcessing.h:1757-1775); a missing
    // column reads as 0 (BlockSetValue), so every product is 0 and nothing is added
    if (!gargs->aggr_idx1 || !gargs->aggr_idx2) return MB_OK;
    a.aggr[0] = gargs->aggr_idx1;
    a.aggr[1] = gargs->aggr_idx2;
    a.agg_op = MB_AGG_MUL;
    a.total_val = 1;
    a.res_layout = MB_RES_SCALAR;
    a.res = res + 4;
  }
  a.count_after = -1;
  if (gpuCache != nullptr) {
    a.gpu_cache = gpuCache;
    a.segment_group = segment_group;
    a.start_offset = start_offset;
    a.segment_size = 1 << 20;  // SEGMENT_SIZE (src/gpudb/common.h:73)
  }
  return launch_star(&a, static_cast<cudaStream_t>(stream), 0);
}

int mb_filter_probe_group_by_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_probeArgsGPU* pargs,
                                  const mb_groupbyArgsGPU* gargs, int num_tuples, int* res, int start_offset,
                                  const short* segment_group, mb_stream_t stream) {
  if (pargs == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, nullptr, fargs, pargs, gargs, num_tuples, res, start_offset, segment_group, stream,
                     true, false);
}

int mb_probe_group_by_GPU2(const int* gpuCache, const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs,
                           int num_tuples, int* res, int start_offset, const short* segment_group, mb_stream_t stream) {
  if (pargs == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, nullptr, nullptr, pargs, gargs, num_tuples, res, start_offset, segment_group, stream,
                     true, false);
}

int mb_filter_probe_aggr_GPU2(const int* gpuCache, const mb_filterArgsGPU* fargs, const mb_probeArgsGPU* pargs,
                              const mb_groupbyArgsGPU* gargs, int num_tuples, int* res, int start_offset,
                              const short* segment_group, mb_stream_t stream) {
  if (pargs == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, nullptr, fargs, pargs, gargs, num_tuples, res, start_offset, segment_group, stream,
                     false, true);
}

int mb_probe_aggr_GPU2(const int* gpuCache, const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs,
                       int num_tuples, int* res, int start_offset, const short* segment_group, mb_stream_t stream) {
  if (pargs == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, nullptr, nullptr, pargs, gargs, num_tuples, res, start_offset, segment_group, stream,
                     false, true);
}

int mb_filter_probe_group_by_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_filterArgsGPU* fargs,
                                  const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs, int num_tuples,
                                  int* res, mb_stream_t stream) {
  if (offset == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, offset, fargs, pargs, gargs, num_tuples, res, 0, nullptr, stream, true, false);
}

int mb_probe_group_by_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_probeArgsGPU* pargs,
                           const mb_groupbyArgsGPU* gargs, int num_tuples, int* res, mb_stream_t stream) {
  if (offset == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, offset, nullptr, pargs, gargs, num_tuples, res, 0, nullptr, stream, true, false);
}

int mb_groupByGPU(const int* gpuCache, const mb_offsetGPU* offset, const mb_groupbyArgsGPU* gargs, int num_tuples,
                  int* res, mb_stream_t stream) {
  if (offset == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, offset, nullptr, nullptr, gargs, num_tuples, res, 0, nullptr, stream, true, false);
}

int mb_aggregationGPU(const int* gpuCache, const int* lo_off, const mb_groupbyArgsGPU* gargs, int num_tuples,
                      int* res, mb_stream_t stream) {
  mb_offsetGPU off = {const_cast<int*>(lo_off), nullptr, nullptr, nullptr, nullptr};
  if (lo_off == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, &off, nullptr, nullptr, gargs, num_tuples, res, 0, nullptr, stream, false, false);
}

int mb_probe_aggr_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_probeArgsGPU* pargs,
                       const mb_groupbyArgsGPU* gargs, int num_tuples, int* res, mb_stream_t stream) {
  if (offset == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, offset, nullptr, pargs, gargs, num_tuples, res, 0, nullptr, stream, false, true);
}

int mb_filter_probe_aggr_GPU3(const int* gpuCache, const mb_offsetGPU* offset, const mb_filterArgsGPU* fargs,
                              const mb_probeArgsGPU* pargs, const mb_groupbyArgsGPU* gargs, int num_tuples, int* res,
                              mb_stream_t stream) {
  if (offset == nullptr) return MB_ERR_ARG;
  return engine_star(gpuCache, offset, fargs, pargs, gargs, num_tuples, res, 0, nullptr, stream, false, true,
                     kEngineSecondFilter);
}

// ---- generator ----------------------------------------------------------------------------
int mb_gen_fact_column(int col, uint64_t seed, int64_t row0, int64_t n, int s_len, int c_len, int p_len, int* out,
                       mb_stream_t stream) {
  if (!mb_is_fact_column(col) || n < 0 || row0 < 0) return MB_ERR_ARG;
  if (n == 0) return MB_OK;
  if (out == nullptr) return MB_ERR_ARG;
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  if (n == 0) return MB_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > ds->num_sms * 16) blocks = ds->num_sms * 16;
  gen_fact_kernel<<<static_cast<int>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      col, seed, row0, n, s_len, c_len, p_len, out);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

int mb_gen_dim_column(int col, uint64_t seed, int64_t n, int* out, mb_stream_t stream) {
  if (mb_is_fact_column(col) || n < 0) return MB_ERR_ARG;
  if (n == 0) return MB_OK;
  if (out == nullptr) return MB_ERR_ARG;
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  if (ds == nullptr) return err;
  if (n == 0) return MB_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > ds->num_sms * 16) blocks = ds->num_sms * 16;
  gen_dim_kernel<<<static_cast<int>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(col, seed, n, out);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

int mb_gen_fact_column_host(int col, uint64_t seed, int64_t row0, int64_t n, int s_len, int c_len, int p_len,
                            int* out, int nthreads) {
  if (!mb_is_fact_column(col) || n < 0 || row0 < 0) return MB_ERR_ARG;
  if (n == 0) return MB_OK;
  if (out == nullptr) return MB_ERR_ARG;
  host_parallel(n, nthreads, [&](long long lo, long long hi) {
    for (long long i = lo; i < hi; ++i)
      out[i] = mb_gen_fact_value(seed, col, static_cast<uint64_t>(row0 + i), s_len, c_len, p_len);
  });
  return MB_OK;
}

int mb_gen_dim_column_host(int col, uint64_t seed, int64_t n, int* out, int nthreads) {
  if (mb_is_fact_column(col) || n < 0) return MB_ERR_ARG;
  if (n == 0) return MB_OK;
  if (out == nullptr) return MB_ERR_ARG;
  host_parallel(n, nthreads, [&](long long lo, long long hi) {
    for (long long i = lo; i < hi; ++i) out[i] = mb_gen_dim_value(seed, col, static_cast<uint64_t>(i));
  });
  return MB_OK;
}

}  // extern "C"
