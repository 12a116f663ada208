// ref_driver.cpp — runs the reference's own standalone CPU engine (src/cpu/ssb/q11.cpp,
// q21.cpp, q41.cpp, compiled unmodified from the reference tree with the tbb shim) on
// seeded synthetic tables. TEST INFRASTRUCTURE ONLY: it pins the oracle to the
// reference's code and times the reference's CPU path for the baseline arm.
//
// The reference's runQuery prints its result ("Revenue: N" or "year key sum" rows and
// "Res Count: N"); this driver adds one JSON line per trial: {"trial": i, "ms": t}.
//
// usage: ref_qNN SEED LO_LEN S_LEN C_LEN P_LEN D_LEN TRIALS
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../mordred_b200/csrc/ssbgen.h"

#if REF_QUERY == 11
float runQuery(int* lo_orderdate, int* lo_discount, int* lo_quantity, int* lo_extendedprice, int num_items);
#elif REF_QUERY == 21
float runQuery(int* lo_orderdate, int* lo_partkey, int* lo_suppkey, int* lo_revenue, int lo_len, int* p_partkey,
               int* p_brand1, int* p_category, int p_len, int* d_datekey, int* d_year, int d_len, int* s_suppkey,
               int* s_region, int s_len);
#elif REF_QUERY == 41
float runQuery(int* lo_orderdate, int* lo_custkey, int* lo_partkey, int* lo_suppkey, int* lo_revenue,
               int* lo_supplycost, int lo_len, int* d_datekey, int* d_year, int d_len, int* p_partkey, int* p_mfgr,
               int p_len, int* s_suppkey, int* s_region, int s_len, int* c_custkey, int* c_region, int* c_nation,
               int c_len);
#else
#error "REF_QUERY must be 11, 21 or 41"
#endif

static std::vector<int> fact(int col, uint64_t seed, long n, int s, int c, int p) {
  std::vector<int> v(static_cast<size_t>(n));
  for (long i = 0; i < n; ++i) v[i] = mb_gen_fact_value(seed, col, static_cast<uint64_t>(i), s, c, p);
  return v;
}

static std::vector<int> dim(int col, uint64_t seed, long n) {
  std::vector<int> v(static_cast<size_t>(n));
  for (long i = 0; i < n; ++i) v[i] = mb_gen_dim_value(seed, col, static_cast<uint64_t>(i));
  return v;
}

int main(int argc, char** argv) {
  if (argc < 8) {
    std::fprintf(stderr, "usage: %s SEED LO_LEN S_LEN C_LEN P_LEN D_LEN TRIALS\n", argv[0]);
    return 2;
  }
  const uint64_t seed = std::strtoull(argv[1], nullptr, 10);
  const long lo_len = std::atol(argv[2]);
  const int s_len = std::atoi(argv[3]), c_len = std::atoi(argv[4]), p_len = std::atoi(argv[5]);
  const int d_len = std::atoi(argv[6]), trials = std::atoi(argv[7]);
#if REF_QUERY == 11
  auto od = fact(MB_LO_ORDERDATE, seed, lo_len, s_len, c_len, p_len);
  auto disc = fact(MB_LO_DISCOUNT, seed, lo_len, s_len, c_len, p_len);
  auto qty = fact(MB_LO_QUANTITY, seed, lo_len, s_len, c_len, p_len);
  auto price = fact(MB_LO_EXTENDEDPRICE, seed, lo_len, s_len, c_len, p_len);
  for (int t = 0; t < trials; ++t) {
    float ms = runQuery(od.data(), disc.data(), qty.data(), price.data(), static_cast<int>(lo_len));
    std::printf("{\"trial\": %d, \"ms\": %f}\n", t, ms);
  }
#else
  auto od = fact(MB_LO_ORDERDATE, seed, lo_len, s_len, c_len, p_len);
  auto pk = fact(MB_LO_PARTKEY, seed, lo_len, s_len, c_len, p_len);
  auto sk = fact(MB_LO_SUPPKEY, seed, lo_len, s_len, c_len, p_len);
  auto rev = fact(MB_LO_REVENUE, seed, lo_len, s_len, c_len, p_len);
  auto d_datekey = dim(MB_D_DATEKEY, seed, d_len);
  auto d_year = dim(MB_D_YEAR, seed, d_len);
  auto p_partkey = dim(MB_P_PARTKEY, seed, p_len);
  auto s_suppkey = dim(MB_S_SUPPKEY, seed, s_len);
  auto s_region = dim(MB_S_REGION, seed, s_len);
#if REF_QUERY == 21
  auto p_brand1 = dim(MB_P_BRAND1, seed, p_len);
  auto p_category = dim(MB_P_CATEGORY, seed, p_len);
  for (int t = 0; t < trials; ++t) {
    float ms = runQuery(od.data(), pk.data(), sk.data(), rev.data(), static_cast<int>(lo_len), p_partkey.data(),
                        p_brand1.data(), p_category.data(), p_len, d_datekey.data(), d_year.data(), d_len,
                        s_suppkey.data(), s_region.data(), s_len);
    std::printf("{\"trial\": %d, \"ms\": %f}\n", t, ms);
  }
#else
  auto ck = fact(MB_LO_CUSTKEY, seed, lo_len, s_len, c_len, p_len);
  auto cost = fact(MB_LO_SUPPLYCOST, seed, lo_len, s_len, c_len, p_len);
  auto p_mfgr = dim(MB_P_MFGR, seed, p_len);
  auto c_custkey = dim(MB_C_CUSTKEY, seed, c_len);
  auto c_region = dim(MB_C_REGION, seed, c_len);
  auto c_nation = dim(MB_C_NATION, seed, c_len);
  for (int t = 0; t < trials; ++t) {
    float ms = runQuery(od.data(), ck.data(), pk.data(), sk.data(), rev.data(), cost.data(), static_cast<int>(lo_len),
                        d_datekey.data(), d_year.data(), d_len, p_partkey.data(), p_mfgr.data(), p_len,
                        s_suppkey.data(), s_region.data(), s_len, c_custkey.data(), c_region.data(), c_nation.data(),
                        c_len);
    std::printf("{\"trial\": %d, \"ms\": %f}\n", t, ms);
  }
#endif
#endif
  std::fflush(stdout);
  return 0;
}
