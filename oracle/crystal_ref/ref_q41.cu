// Test infrastructure: the reference's own src/ssb/q41.cu, compiled unmodified against
// include/crystal_b200.cuh (its main() is renamed and never called), with launchers that
// run its build and probe kernels <128, 4> the way its runQuery does.
// (its main() names CUB's CommandLineArgs without including CUB's test header)
#include "cub/test/test_util.h"
#define main reference_q41_main
#include "q41.cu"
#undef main

extern "C" int crystal_ref_q41(int* lo_orderdate, int* lo_custkey, int* lo_partkey, int* lo_suppkey, int* lo_revenue,
                               int* lo_supplycost, int lo_len, int* d_datekey, int* d_year, int d_len, int* p_partkey,
                               int* p_mfgr, int p_len, int* s_suppkey, int* s_region, int s_len, int* c_custkey,
                               int* c_region, int* c_nation, int c_len, int d_val_len, int* ht_s, int* ht_c,
                               int* ht_p, int* ht_d, int* res) {
  const int tile_items = 128 * 4;
  build_hashtable_s<128, 4><<<(s_len + tile_items - 1) / tile_items, 128>>>(s_region, s_suppkey, s_len, ht_s, s_len);
  build_hashtable_c<128, 4><<<(c_len + tile_items - 1) / tile_items, 128>>>(c_region, c_custkey, c_nation, c_len,
                                                                           ht_c, c_len);
  build_hashtable_p<128, 4><<<(p_len + tile_items - 1) / tile_items, 128>>>(p_mfgr, p_partkey, p_len, ht_p, p_len);
  build_hashtable_d<128, 4><<<(d_len + tile_items - 1) / tile_items, 128>>>(d_datekey, d_year, d_len, ht_d, d_val_len,
                                                                           19920101);
  probe<128, 4><<<(lo_len + tile_items - 1) / tile_items, 128>>>(lo_orderdate, lo_partkey, lo_custkey, lo_suppkey,
                                                                 lo_revenue, lo_supplycost, lo_len, ht_p, p_len, ht_s,
                                                                 s_len, ht_c, c_len, ht_d, d_val_len, res);
  cudaError_t e = cudaGetLastError();
  return static_cast<int>(e == cudaSuccess ? cudaDeviceSynchronize() : e);
}
