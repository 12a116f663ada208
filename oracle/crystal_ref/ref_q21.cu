// Test infrastructure: the reference's own src/ssb/q21.cu, compiled unmodified against
// include/crystal_b200.cuh (its main() is renamed and never called), with launchers that
// run its build and probe kernels <128, 4> the way its runQuery does.
#define main reference_q21_main
#include "q21.cu"
#undef main

extern "C" int crystal_ref_q21(int* lo_orderdate, int* lo_partkey, int* lo_suppkey, int* lo_revenue, int lo_len,
                               int* p_partkey, int* p_brand1, int* p_category, int p_len, int* d_datekey,
                               int* d_year, int d_len, int* s_suppkey, int* s_region, int s_len, int d_val_len,
                               int* ht_s, int* ht_p, int* ht_d, int* res) {
  const int tile_items = 128 * 4;
  build_hashtable_s<128, 4><<<(s_len + tile_items - 1) / tile_items, 128>>>(s_region, s_suppkey, s_len, ht_s, s_len);
  build_hashtable_p<128, 4><<<(p_len + tile_items - 1) / tile_items, 128>>>(p_category, p_partkey, p_brand1, p_len,
                                                                           ht_p, p_len);
  build_hashtable_d<128, 4><<<(d_len + tile_items - 1) / tile_items, 128>>>(d_datekey, d_year, d_len, ht_d, d_val_len,
                                                                           19920101);
  probe<128, 4><<<(lo_len + tile_items - 1) / tile_items, 128>>>(lo_orderdate, lo_partkey, lo_suppkey, lo_revenue,
                                                                 lo_len, ht_s, s_len, ht_p, p_len, ht_d, d_val_len,
                                                                 res);
  cudaError_t e = cudaGetLastError();
  return static_cast<int>(e == cudaSuccess ? cudaDeviceSynchronize() : e);
}
