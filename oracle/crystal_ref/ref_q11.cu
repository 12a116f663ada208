// Test infrastructure: the reference's own src/ssb/q11.cu, compiled unmodified against
// include/crystal_b200.cuh (its main() is renamed and never called), with a launcher that
// runs its QueryKernel<128, 4> the way its runQuery does.
#define main reference_q11_main
#include "q11.cu"
#undef main

extern "C" int crystal_ref_q11(int* lo_orderdate, int* lo_discount, int* lo_quantity, int* lo_extendedprice, int n,
                               unsigned long long* revenue, int* d_total) {
  const int tile_items = 128 * 4;
  QueryKernel<128, 4><<<(n + tile_items - 1) / tile_items, 128>>>(lo_orderdate, lo_discount, lo_quantity,
                                                                   lo_extendedprice, n, revenue, d_total);
  cudaError_t e = cudaGetLastError();
  return static_cast<int>(e == cudaSuccess ? cudaDeviceSynchronize() : e);
}
