/*
 * ssbgen.h — seeded, counter-based generator for the synthetic star-schema tables.
 *
 * Header-only and usable from nvcc (host and device) and from plain gcc/g++, so the
 * GPU generator, the host generator and any CPU-side driver produce bit-identical
 * columns from the same (seed, column, row) triple without sharing state.
 *
 * Shapes and encodings follow the star schema the engine runs on (the reference
 * loader's encodings, test/ssb/loader/convert.py:53-96):
 *   fact     lo_orderdate  yyyymmdd of a day drawn uniformly from 1992-01-01..1998-12-31
 *            lo_quantity   U{1..50}         lo_discount    U{0..10}
 *            lo_extendedprice U{90100..10494950}
 *            lo_suppkey    U{1..S}  lo_custkey U{1..C}  lo_partkey U{1..P}   (dense 1-based keys)
 *            lo_revenue    U{90100..10494950}  lo_supplycost U{54000..600000}
 *   date     2,557 rows, d_datekey = yyyymmdd, d_year, d_yearmonthnum = yyyymm
 *   supplier/customer  key = row+1, city U{0..249}, nation = city/10, region = nation/5
 *   part     key = row+1, brand1 U{0..999}, category = brand1/40, mfgr = category/5
 * Keys are 1-based because a zero key marks an empty slot in the perfect hash tables.
 */
#ifndef MORDRED_B200_SSBGEN_H
#define MORDRED_B200_SSBGEN_H

#include <stdint.h>

#if defined(__CUDACC__)
#define MB_HD __host__ __device__ __forceinline__
#else
#define MB_HD static inline
#endif

/* Column identifiers; each owns an independent random stream. */
enum mb_gen_column {
  MB_LO_ORDERDATE = 0,
  MB_LO_QUANTITY = 1,
  MB_LO_DISCOUNT = 2,
  MB_LO_EXTENDEDPRICE = 3,
  MB_LO_SUPPKEY = 4,
  MB_LO_CUSTKEY = 5,
  MB_LO_PARTKEY = 6,
  MB_LO_REVENUE = 7,
  MB_LO_SUPPLYCOST = 8,
  MB_D_DATEKEY = 16,
  MB_D_YEAR = 17,
  MB_D_YEARMONTHNUM = 18,
  MB_S_SUPPKEY = 32,
  MB_S_CITY = 33,
  MB_S_NATION = 34,
  MB_S_REGION = 35,
  MB_C_CUSTKEY = 48,
  MB_C_CITY = 49,
  MB_C_NATION = 50,
  MB_C_REGION = 51,
  MB_P_PARTKEY = 64,
  MB_P_BRAND1 = 65,
  MB_P_CATEGORY = 66,
  MB_P_MFGR = 67
};

#define MB_NUM_DAYS 2557          /* 1992-01-01 .. 1998-12-31 inclusive */
#define MB_DAY0_EPOCH 8035        /* days from 1970-01-01 to 1992-01-01 */
#define MB_FIRST_DATEKEY 19920101
#define MB_LAST_DATEKEY 19981231

/* splitmix64 finaliser (Steele, Lea, Flood 2014). */
MB_HD uint64_t mb_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

/* 64 random bits for (seed, column stream, row). */
MB_HD uint64_t mb_rand64(uint64_t seed, uint32_t stream, uint64_t row) {
  uint64_t base = mb_mix64(seed + 0x9e3779b97f4a7c15ULL * (uint64_t)(stream + 1));
  return mb_mix64(base + 0xd1b54a32d192ed03ULL * (row + 1));
}

/* Uniform integer in [lo, hi] (hi - lo < 2^32) by a 32x32 multiply-shift of the high word. */
MB_HD int32_t mb_uniform(uint64_t seed, uint32_t stream, uint64_t row, int32_t lo, int32_t hi) {
  uint64_t r = mb_rand64(seed, stream, row) >> 32;
  uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo + 1);
  return (int32_t)((int64_t)lo + (int64_t)((r * span) >> 32));
}

/* Proleptic Gregorian date of a day number counted from 1970-01-01, as yyyymmdd
 * (the era/day-of-era construction published by H. Hinnant, "chrono-compatible
 * low-level date algorithms"). */
MB_HD int32_t mb_yyyymmdd_from_epoch_day(int32_t z) {
  z += 719468;
  int32_t era = (z >= 0 ? z : z - 146096) / 146097;
  int32_t doe = z - era * 146097;
  int32_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  int32_t y = yoe + era * 400;
  int32_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  int32_t mp = (5 * doy + 2) / 153;
  int32_t d = doy - (153 * mp + 2) / 5 + 1;
  int32_t m = mp < 10 ? mp + 3 : mp - 9;
  y += (m <= 2);
  return y * 10000 + m * 100 + d;
}

/* Date dimension row i (0 <= i < MB_NUM_DAYS) -> yyyymmdd. */
MB_HD int32_t mb_datekey_of_day(int32_t i) { return mb_yyyymmdd_from_epoch_day(MB_DAY0_EPOCH + i); }

/* Value of fact column `col` at `row`. dim sizes give the foreign-key ranges. */
MB_HD int32_t mb_gen_fact_value(uint64_t seed, int col, uint64_t row,
                                int32_t s_len, int32_t c_len, int32_t p_len) {
  switch (col) {
    case MB_LO_ORDERDATE:
      return mb_datekey_of_day(mb_uniform(seed, MB_LO_ORDERDATE, row, 0, MB_NUM_DAYS - 1));
    case MB_LO_QUANTITY: return mb_uniform(seed, MB_LO_QUANTITY, row, 1, 50);
    case MB_LO_DISCOUNT: return mb_uniform(seed, MB_LO_DISCOUNT, row, 0, 10);
    case MB_LO_EXTENDEDPRICE: return mb_uniform(seed, MB_LO_EXTENDEDPRICE, row, 90100, 10494950);
    case MB_LO_SUPPKEY: return mb_uniform(seed, MB_LO_SUPPKEY, row, 1, s_len);
    case MB_LO_CUSTKEY: return mb_uniform(seed, MB_LO_CUSTKEY, row, 1, c_len);
    case MB_LO_PARTKEY: return mb_uniform(seed, MB_LO_PARTKEY, row, 1, p_len);
    case MB_LO_REVENUE: return mb_uniform(seed, MB_LO_REVENUE, row, 90100, 10494950);
    case MB_LO_SUPPLYCOST: return mb_uniform(seed, MB_LO_SUPPLYCOST, row, 54000, 600000);
    default: return 0;
  }
}

/* Value of dimension column `col` at `row`. */
MB_HD int32_t mb_gen_dim_value(uint64_t seed, int col, uint64_t row) {
  switch (col) {
    case MB_D_DATEKEY: return mb_datekey_of_day((int32_t)row);
    case MB_D_YEAR: return mb_datekey_of_day((int32_t)row) / 10000;
    case MB_D_YEARMONTHNUM: return mb_datekey_of_day((int32_t)row) / 100;
    case MB_S_SUPPKEY: case MB_C_CUSTKEY: case MB_P_PARTKEY: return (int32_t)row + 1;
    case MB_S_CITY: return mb_uniform(seed, MB_S_CITY, row, 0, 249);
    case MB_S_NATION: return mb_uniform(seed, MB_S_CITY, row, 0, 249) / 10;
    case MB_S_REGION: return mb_uniform(seed, MB_S_CITY, row, 0, 249) / 50;
    case MB_C_CITY: return mb_uniform(seed, MB_C_CITY, row, 0, 249);
    case MB_C_NATION: return mb_uniform(seed, MB_C_CITY, row, 0, 249) / 10;
    case MB_C_REGION: return mb_uniform(seed, MB_C_CITY, row, 0, 249) / 50;
    case MB_P_BRAND1: return mb_uniform(seed, MB_P_BRAND1, row, 0, 999);
    case MB_P_CATEGORY: return mb_uniform(seed, MB_P_BRAND1, row, 0, 999) / 40;
    case MB_P_MFGR: return mb_uniform(seed, MB_P_BRAND1, row, 0, 999) / 200;
    default: return 0;
  }
}

MB_HD int mb_is_fact_column(int col) { return col >= 0 && col < 16; }

#endif /* MORDRED_B200_SSBGEN_H */
