// noalloc.cu — the Query B probe for callers that cannot allocate device memory.
//
// The ordinary entry points keep their device scratch (the status word kernels report
// into) in memory the library cudaMalloc's on the first call on a device. Some callers
// cannot let a library do that: an executor that carves every device buffer out of an
// arena it sized up front (as the reference's segment cache does with its bump
// allocators) cannot have a call grow the device footprint behind its accounting, and a
// serving thread cannot take cudaMalloc's device-wide synchronisation in the middle of
// other streams' work. mb_q41_probe_noalloc serves them: it keeps its scratch — the
// status word and the presence bitmap of the supplier table — in the file-scope array
// below and allocates nothing, in this file or in anything it calls.
#include <cstring>
#include <mutex>

#include "star.cuh"

namespace mb {

// Scratch layout (32-bit words): [0] status bits of the current call, [1, 64) padding,
// [64, 64 + 8,192) presence bitmap of the supplier table (up to 262,144 slots).
constexpr int kNoAllocBitmapWord = 64;
constexpr int kNoAllocMaxSupplierSlots = 262144;
constexpr int kNoAllocWords = kNoAllocBitmapWord + kNoAllocMaxSupplierSlots / 32;

// 33,024 bytes on every device that loads the library, held until the process exits.
// In host code this name is only a host-side stand-in for the device symbol, never a
// device address: host code uses the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned int g_noalloc_scratch[kNoAllocWords];

// Clears the status word and writes the presence bitmap of an MB_HT_KEY table
// (bit s set iff ht[s] != 0) into the scratch.
__global__ void noalloc_presence_kernel(const int* ht, int slots) {
  if (blockIdx.x == 0 && threadIdx.x == 0) g_noalloc_scratch[0] = 0;
  const int words = (slots + 31) / 32;
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    uint32_t word = 0;
    for (int j = 0; j < 32; ++j) {
      const int s = w * 32 + j;
      if (s < slots && __ldg(ht + s) != 0) word |= 1u << j;
    }
    g_noalloc_scratch[kNoAllocBitmapWord + w] = word;
  }
}

struct NoAllocDevice {
  bool ready = false;
  DeviceState ds;              // ds.status points at word 0 of the scratch
  unsigned int* scratch = nullptr;
};

static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc[64];

// Once per device, with that device current: device limits, kernel attributes and the
// scratch's device address. None of these calls allocates device memory.
static int noalloc_setup(NoAllocDevice** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MB_ERR_NODEV;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc[dev];
  if (!d.ready) {
    int sms = 0, optin = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MB_ERR_NODEV;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      return MB_ERR_NODEV;
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) return MB_ERR_CUDA;
    d.scratch = static_cast<unsigned int*>(ptr);
    d.ds.device = dev;
    d.ds.num_sms = sms;
    d.ds.max_smem_optin = optin;
    d.ds.status = d.scratch;
    const int e = star_init_device(d.ds);
    if (e != MB_OK) return e;
    d.ready = true;
  }
  *out = &d;
  return MB_OK;
}

}  // namespace mb

using namespace mb;

extern "C" int mb_q41_probe_noalloc(const int* lo_orderdate, const int* lo_partkey, const int* lo_custkey,
                                    const int* lo_suppkey, const int* lo_revenue, const int* lo_supplycost, int lo_len,
                                    const int* ht_p, int p_len, const int* ht_s, int s_len, const int* ht_c, int c_len,
                                    const int* ht_d, int d_len, int* res, unsigned int* status, mb_stream_t stream) {
  if (s_len > kNoAllocMaxSupplierSlots) return MB_ERR_SIZE;  // the scratch bitmap holds 262,144 slots
  if (lo_len < 0 || s_len <= 0 || ht_s == nullptr) return MB_ERR_ARG;
  NoAllocDevice* d = nullptr;
  int e = noalloc_setup(&d);
  if (e != MB_OK) return e;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  const int words = (s_len + 31) / 32;
  const int blocks = (words + 255) / 256 < d->ds.num_sms ? (words + 255) / 256 : d->ds.num_sms;
  noalloc_presence_kernel<<<blocks, 256, 0, st>>>(ht_s, s_len);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);

  // the same pipeline as mb_q41_probe (src/ssb/q41.cu:50-62), with the supplier
  // presence read from the scratch instead of derived from the table in every CTA
  mb_star_args a;
  memset(&a, 0, sizeof(a));
  a.num_rows = lo_len;
  a.num_probes = 4;
  a.probe[0] = {lo_suppkey, ht_s, s_len, 0, MB_HT_KEY, 0, 0, -1, d->scratch + kNoAllocBitmapWord};
  a.probe[1] = {lo_custkey, ht_c, c_len, 0, MB_HT_KEY_VAL, 0, 7, 1, nullptr};
  a.probe[2] = {lo_partkey, ht_p, p_len, 0, MB_HT_KEY, 0, 0, -1, nullptr};
  a.probe[3] = {lo_orderdate, ht_d, d_len, 19920101, MB_HT_KEY_VAL, 1992, 1, 0, nullptr};
  a.aggr[0] = lo_revenue;
  a.aggr[1] = lo_supplycost;
  a.agg_op = MB_AGG_SUB;
  a.total_val = (1998 - 1992 + 1) * 25;
  a.res_layout = MB_RES_CRYSTAL4;
  a.res = res;
  a.count_after = -1;
  e = launch_star(&a, st, 0, &d->ds);
  if (e != MB_OK) return e;
  if (status != nullptr &&
      cudaMemcpyAsync(status, d->scratch, sizeof(unsigned int), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MB_ERR_CUDA;
  return MB_OK;
}
