// common.cuh — shared device helpers for the sm_100a kernels: bulk-copy (TMA) and
// mbarrier PTX wrappers, bounded waits, the per-device status word and launch accounting.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mordred_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 900)
#error "mordred_b200 kernels target sm_100a (cp.async.bulk and mbarrier tx-counts)"
#endif

namespace mb {

static __device__ __noinline__ int slow_mod(int d, int m) { return d % m; }

// ((key - key_min) % slots) in 32-bit two's complement (crystal/join.cuh:3). Keys in
// [key_min, key_min + slots) map to themselves and the next range wraps by one
// subtraction (a dense 1-based key N lands on slot 0); only other keys divide.
__device__ __forceinline__ int pht_slot(int key, int slots, int kmin) {
  const int d = static_cast<int>(static_cast<unsigned>(key) - static_cast<unsigned>(kmin));
  if (static_cast<unsigned>(d) < static_cast<unsigned>(slots)) return d;
  if (static_cast<unsigned>(d) < 2u * static_cast<unsigned>(slots) && slots <= (1 << 30)) return d - slots;
  return slow_mod(d, slots);
}

// Longest a CTA waits on one bulk-copy stage before it gives up, sets
// MB_STATUS_TIMEOUT and returns (a healthy copy lands in microseconds).
constexpr unsigned long long kWaitLimitNs = 4000000000ull;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Test phase `parity` of `bar`; a waiting thread is suspended until the phase completes
// or the hint (ns) elapses, so a warp waiting for a tile does not spin through issue slots.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar` to complete, for at most kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kWaitLimitNs) return false;
  }
}

// L2 policy: fact-column tiles are read once, so they are marked evict-first and the
// hash tables probed alongside them keep their L2 residency.
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar` (no multicast).
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
      "[%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ int4 lds128(const int* p) {
  return *reinterpret_cast<const int4*>(p);
}

// Read-only 8-byte hash-table slot through the non-coherent path.
__device__ __forceinline__ unsigned long long ldg_u64(const int* p) {
  return __ldg(reinterpret_cast<const unsigned long long*>(p));
}

__device__ __forceinline__ void set_status(unsigned int* status, unsigned int bits) {
  if (status) atomicOr(status, bits);
}

}  // namespace mb

// ---- host side -----------------------------------------------------------------
namespace mb {

// Per-device runtime state: the status word kernels report into, SM count and smem
// limits. Created once per device by mb_init (or the first launch).
struct DeviceState {
  int device = -1;
  int num_sms = 0;
  int max_smem_optin = 0;
  unsigned int* status = nullptr;  // device word, cudaMalloc'd at init
};

// Returns nullptr (and sets *err) if the current device cannot be initialised.
DeviceState* current_device_state(int* err);
void note_launches(unsigned long long n);

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? MB_OK : MB_ERR_CUDA; }

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
inline bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

}  // namespace mb
