/*
 * star_oracle.c — CPU oracle for the star-query hot path (see star_oracle.h).
 * TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline, never the product.
 *
 * Integer semantics are kept exactly: products and differences are formed in 32-bit
 * two's complement (as the reference's int arithmetic on its targets) and then
 * sign-extended into 64-bit sums; hashes use C's truncating %, and a negative slot or
 * group index (an out-of-bounds access in the reference) is reported as a status bit
 * and the row skipped instead of being written out of bounds.
 */
#define _GNU_SOURCE
#include "star_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

static int orc_threads(int n) {
  if (n > 0) return n;
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

static inline int i32_mul(int a, int b) { return (int)((unsigned)a * (unsigned)b); }
static inline int i32_sub(int a, int b) { return (int)((unsigned)a - (unsigned)b); }
static inline unsigned long long widen(int v) { return (unsigned long long)(long long)v; }

/* ((X - Z) % Y) of crystal/join.cuh:3, evaluated in 32-bit ints. */
static inline int pht_slot(int key, int slots, int kmin) { return i32_sub(key, kmin) % slots; }

typedef void (*orc_range_fn)(void* ctx, int tid, int64_t lo, int64_t hi);

typedef struct {
  orc_range_fn fn;
  void* ctx;
  int tid;
  int64_t lo, hi;
} orc_job;

static void* orc_job_main(void* p) {
  orc_job* j = (orc_job*)p;
  j->fn(j->ctx, j->tid, j->lo, j->hi);
  return NULL;
}

/* Split [0, n) into nthreads contiguous ranges, one thread each. */
static void orc_parallel(int64_t n, int nthreads, orc_range_fn fn, void* ctx) {
  if (nthreads < 1) nthreads = 1;
  if (n < 4096) nthreads = 1;
  orc_job* jobs = (orc_job*)calloc((size_t)nthreads, sizeof(orc_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  int64_t chunk = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
    jobs[t].tid = t;
    jobs[t].lo = t * chunk < n ? t * chunk : n;
    jobs[t].hi = (t + 1) * chunk < n ? (t + 1) * chunk : n;
  }
  for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, orc_job_main, &jobs[t]);
  orc_job_main(&jobs[0]);
  for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
}

/* ------------------------------------------------------------------------------- */
/* Engine-style generic pipeline (CPUProcessing.cu:723-866)                          */
/* ------------------------------------------------------------------------------- */

static int rec_ints(int layout) { return layout == 1 ? 6 : layout == 2 ? 4 : 2; }
static int rec_sum_off(int layout) { return layout == 1 ? 4 : layout == 2 ? 2 : 0; }

typedef struct {
  const orc_star_args* a;
  int* priv;                 /* per thread: total_val records of rec_ints ints */
  unsigned char* touched;    /* per thread: total_val flags */
  unsigned long long* sum;   /* per thread scalar */
  unsigned long long* cnt;   /* per thread count */
  unsigned* status;          /* per thread */
} star_ctx;

/* Physical row visited at position r of the call: the offset list, the segment mapping
 * (CPUProcessing.cu:741,751) or r itself. */
static inline int64_t visit_row(const orc_star_args* a, int64_t r) {
  if (a->rows) return a->rows[r];
  if (a->segment_size > 0) {
    const int64_t S = a->segment_size;
    const int64_t seg = a->segment_group ? (int64_t)a->segment_group[r / S] : (a->start_offset + r) / S;
    return seg * S + r % S;
  }
  return r;
}

/* Filters, then probes in order, of the row at position r (physical row `row`), as
 * filter_probe_group_by_CPU / _CPU2 (CPUProcessing.cu:723-1032). Returns 1 when the row
 * passes; gv[p] = probe p's payload, out[p] = its selection output (VAL_OFF: the
 * dimension row, KEY_VAL: the payload, KEY: 0, pass-through: the passed offset).
 * *cnt counts rows per count_after. */
static int eval_row(const orc_star_args* a, int64_t r, int64_t row, int* gv, int* out, unsigned* status,
                    unsigned long long* cnt) {
  for (int f = 0; f < a->num_filters; ++f) {
    if (a->count_after == f) ++*cnt;
    const int x = a->filter[f].col[row];
    const int m = a->filter[f].mode, c1 = a->filter[f].c1, c2 = a->filter[f].c2;
    const int ok = m == 1 ? (x >= c1 && x <= c2) : m == 0 ? (x == c1) : (x == c1 || x == c2);
    if (!ok) return 0;
  }
  if (a->count_after >= a->num_filters) ++*cnt;
  for (int p = 0; p < a->num_probes; ++p) {
    const orc_probe* Q = &a->probe[p];
    gv[p] = 0;
    out[p] = 0;
    if (Q->layout == ORC_LAYOUT_PASS) {
      const int d = Q->fkey[r];
      if (d < 0 || d >= Q->num_slots) { *status |= ORC_PROBE_RANGE; return 0; }
      gv[p] = Q->ht[d];
      out[p] = d;
      continue;
    }
    const int h = pht_slot(Q->fkey[row], Q->num_slots, Q->key_min);
    if (h < 0) { *status |= ORC_PROBE_RANGE; return 0; }
    if (Q->layout == 0) {
      if (Q->ht[h] == 0) return 0;
    } else {
      const int lo32 = Q->ht[2 * (int64_t)h], hi32 = Q->ht[2 * (int64_t)h + 1];
      if (Q->layout == 2) {
        /* engine tables: present when the 8-byte slot is nonzero; payload = group value,
           selection output = the dimension row (ht[2h+1] - 1, BlockLibrary.cuh:9-33) */
        if (lo32 == 0 && hi32 == 0) return 0;
        gv[p] = lo32;
        out[p] = hi32 - 1;
      } else {
        if (lo32 == 0 && hi32 == 0) return 0;
        gv[p] = hi32;
        out[p] = hi32;
      }
    }
  }
  if (a->count_after < 0) ++*cnt;
  return 1;
}

static void star_range(void* vctx, int tid, int64_t lo, int64_t hi) {
  star_ctx* C = (star_ctx*)vctx;
  const orc_star_args* a = C->a;
  const int layout = a->res_layout;
  const int R = rec_ints(layout);
  int* priv = C->priv ? C->priv + (size_t)tid * (size_t)a->total_val * (size_t)R : NULL;
  unsigned char* touched = C->touched ? C->touched + (size_t)tid * (size_t)a->total_val : NULL;
  unsigned long long sum = 0, cnt = 0;
  unsigned status = 0;
  for (int64_t r = lo; r < hi; ++r) {
    const int64_t row = visit_row(a, r);
    int gv[ORC_MAX_PROBES] = {0, 0, 0, 0}, out[ORC_MAX_PROBES];
    if (!eval_row(a, r, row, gv, out, &status, &cnt)) continue;
    const int a0 = a->aggr[0][row];
    int v;
    switch (a->agg_op) {
      case 0: v = a0; break;
      case 1: v = i32_sub(a0, a->aggr[1][row]); break;
      case 2: v = i32_mul(a0, a->aggr[1][row]); break;
      default: v = i32_mul(a0, gv[0]); break;
    }
    if (layout == 0) { sum += widen(v); continue; }
    unsigned hh = (unsigned)a->group_bias;
    for (int p = 0; p < a->num_probes; ++p)
      hh += (unsigned)i32_sub(gv[p], a->probe[p].min_val) * (unsigned)a->probe[p].unique_val;
    const int g = (int)hh % a->total_val;
    if (g < 0) { status |= ORC_GROUP_RANGE; continue; }
    int* rec = priv + (size_t)g * R;
    if (layout == 1 || layout == 2)
      for (int p = 0; p < a->num_probes; ++p)
        if (a->probe[p].res_slot >= 0) rec[a->probe[p].res_slot] = gv[p];
    unsigned long long* s = (unsigned long long*)(rec + rec_sum_off(layout));
    *s += widen(v);
    touched[g] = 1;
  }
  C->sum[tid] = sum;
  C->cnt[tid] = cnt;
  C->status[tid] = status;
}

int64_t orc_select(const orc_star_args* a, int* lo_off, int* const* dim_off, int64_t capacity, unsigned* status) {
  unsigned st = 0;
  unsigned long long cnt = 0;
  int64_t k = 0;
  for (int64_t r = 0; r < a->num_rows; ++r) {
    const int64_t row = visit_row(a, r);
    int gv[ORC_MAX_PROBES], out[ORC_MAX_PROBES];
    if (!eval_row(a, r, row, gv, out, &st, &cnt)) continue;
    if (k < capacity) {
      lo_off[k] = (int)row;
      if (dim_off)
        for (int p = 0; p < a->num_probes; ++p)
          if (dim_off[p]) dim_off[p][k] = out[p];
    }
    ++k;
  }
  if (status) *status |= st;
  return k;
}

unsigned orc_star(const orc_star_args* a, int nthreads) {
  nthreads = orc_threads(nthreads);
  if (a->num_rows < 4096) nthreads = 1;
  star_ctx C;
  memset(&C, 0, sizeof(C));
  C.a = a;
  const int layout = a->res_layout, R = rec_ints(layout);
  if (layout != 0) {
    C.priv = (int*)calloc((size_t)nthreads * (size_t)a->total_val * (size_t)R, sizeof(int) + 0);
    C.touched = (unsigned char*)calloc((size_t)nthreads * (size_t)a->total_val, 1);
  }
  C.sum = (unsigned long long*)calloc((size_t)nthreads, sizeof(unsigned long long));
  C.cnt = (unsigned long long*)calloc((size_t)nthreads, sizeof(unsigned long long));
  C.status = (unsigned*)calloc((size_t)nthreads, sizeof(unsigned));
  orc_parallel(a->num_rows, nthreads, star_range, &C);
  unsigned status = 0;
  unsigned long long total = 0, count = 0;
  for (int t = 0; t < nthreads; ++t) {
    status |= C.status[t];
    total += C.sum[t];
    count += C.cnt[t];
  }
  if (layout == 0) {
    *(unsigned long long*)a->res += total;
  } else {
    int* res = (int*)a->res;
    for (int t = 0; t < nthreads; ++t) {
      const int* pr = C.priv + (size_t)t * (size_t)a->total_val * (size_t)R;
      for (int g = 0; g < a->total_val; ++g) {
        if (!C.touched[(size_t)t * a->total_val + g]) continue;
        const int* src = pr + (size_t)g * R;
        int* dst = res + (size_t)g * R;
        if (layout == 1 || layout == 2)
          for (int p = 0; p < a->num_probes; ++p)
            if (a->probe[p].res_slot >= 0) dst[a->probe[p].res_slot] = src[a->probe[p].res_slot];
        *(unsigned long long*)(dst + rec_sum_off(layout)) +=
            *(const unsigned long long*)(src + rec_sum_off(layout));
      }
    }
  }
  if (a->count) *a->count += count;
  free(C.priv);
  free(C.touched);
  free(C.sum);
  free(C.cnt);
  free(C.status);
  return status;
}

unsigned orc_build(const int* filter, int mode, int c1, int c2, const int* key, const int* val, int64_t n,
                   int* ht, int num_slots, int key_min, int layout, int64_t row_base, uint32_t* presence) {
  unsigned status = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (filter) {
      const int x = filter[i];
      int ok = mode == 1 ? (x >= c1 && x <= c2) : mode == 0 ? (x == c1) : (x == c1 || x == c2);
      if (!ok) continue;
    }
    const int k = key[i];
    const int h = pht_slot(k, num_slots, key_min);
    if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
    int present;
    if (layout == 0) {
      if (ht[h] == 0) ht[h] = k; /* atomicCAS(&ht[h], 0, key) */
      present = k != 0;
    } else if (layout == 1) {
      if (ht[2 * (int64_t)h] == 0) ht[2 * (int64_t)h] = k;
      ht[2 * (int64_t)h + 1] = val[i];
      present = k != 0 || val[i] != 0;
    } else {
      if (val && ht[2 * (int64_t)h] == 0) ht[2 * (int64_t)h] = val[i];
      ht[2 * (int64_t)h + 1] = (int)(row_base + i + 1);
      present = 1;
    }
    if (presence && present) presence[h >> 5] |= 1u << (h & 31);
  }
  return status;
}

unsigned orc_build_rows(const int* filter, int mode, int c1, int c2, const int* key, const int* val,
                        const int* rows, int64_t n, int* ht, int num_slots, int key_min, int64_t row_base,
                        int* minmax, int val_min, int val_max) {
  unsigned status = 0;
  int mn = val_max, mx = val_min;  /* the reference's per-task starting values */
  for (int64_t i = 0; i < n; ++i) {
    /* columns are read at the listed dimension row (or at i); the stored row id is that
       row (or row_base + i) */
    const int64_t row = rows ? (int64_t)rows[i] : i;
    const int64_t rowid = rows ? row : row_base + i;
    if (filter) {
      const int x = filter[row];
      const int ok = mode == 1 ? (x >= c1 && x <= c2) : mode == 0 ? (x == c1) : (x == c1 || x == c2);
      if (!ok) continue;
    }
    const int k = key[row];
    if (k < mn) mn = k;
    if (k > mx) mx = k;
    const int h = pht_slot(k, num_slots, key_min);
    if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
    if (val && ht[2 * (int64_t)h] == 0) ht[2 * (int64_t)h] = val[row];
    ht[2 * (int64_t)h + 1] = (int)(rowid + 1);
  }
  if (minmax && n > 0) {
    if (mn < minmax[0]) minmax[0] = mn;
    if (mx > minmax[1]) minmax[1] = mx;
  }
  return status;
}

/* ------------------------------------------------------------------------------- */
/* Standalone CPU engine (src/cpu/ssb)                                              */
/* ------------------------------------------------------------------------------- */

typedef struct {
  const int *od, *disc, *qty, *price;
  int dlo, dhi, klo, khi, qlt;
  unsigned long long* part;
} q11_ctx;

static void q11_range(void* v, int tid, int64_t lo, int64_t hi) {
  q11_ctx* C = (q11_ctx*)v;
  unsigned long long local = 0;
  for (int64_t i = lo; i < hi; ++i) {
    /* q11.cpp:37-46 */
    int flag = C->qty[i] < C->qlt;
    flag = flag && (C->disc[i] >= C->klo && C->disc[i] <= C->khi);
    flag = flag && (C->od[i] > C->dlo && C->od[i] < C->dhi);
    if (flag) local += widen(i32_mul(C->price[i], C->disc[i]));
  }
  C->part[tid] = local;
}

unsigned long long orc_q11(const int* lo_orderdate, const int* lo_discount, const int* lo_quantity,
                           const int* lo_extendedprice, int64_t n, int date_lo_excl, int date_hi_excl, int disc_lo,
                           int disc_hi, int qty_lt, int nthreads) {
  nthreads = orc_threads(nthreads);
  q11_ctx C = {lo_orderdate, lo_discount, lo_quantity, lo_extendedprice, date_lo_excl, date_hi_excl,
               disc_lo, disc_hi, qty_lt, NULL};
  C.part = (unsigned long long*)calloc((size_t)nthreads, sizeof(unsigned long long));
  orc_parallel(n, nthreads, q11_range, &C);
  unsigned long long revenue = 0;
  for (int t = 0; t < nthreads; ++t) revenue += C.part[t];
  free(C.part);
  return revenue;
}

/* Date table build shared by q21/q41 (q21.cpp:62-70): {datekey, year}, no filter. */
static unsigned build_date(const int* d_datekey, const int* d_year, int d_len, int* ht_d, int d_val_len) {
  unsigned status = 0;
  for (int i = 0; i < d_len; ++i) {
    const int h = pht_slot(d_datekey[i], d_val_len, 19920101);
    if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
    ht_d[2 * h] = d_datekey[i];
    ht_d[2 * h + 1] = d_year[i];
  }
  return status;
}


/* Group accumulator shared by q21/q41: per-thread {key0, key1, u64 sum} records plus
 * a touched flag, merged into the caller's array after the threads join. */
typedef struct {
  int num_groups;
  int stride;          /* ints per record in the caller's array (6 for q21, 4 for q41) */
  int* keys;           /* per thread: num_groups x 2 */
  unsigned long long* sums;
  unsigned char* touched;
  unsigned* status;
} grp_acc;

static void grp_init(grp_acc* G, int nthreads, int num_groups, int stride) {
  G->num_groups = num_groups;
  G->stride = stride;
  G->keys = (int*)calloc((size_t)nthreads * num_groups * 2, sizeof(int));
  G->sums = (unsigned long long*)calloc((size_t)nthreads * num_groups, sizeof(unsigned long long));
  G->touched = (unsigned char*)calloc((size_t)nthreads * num_groups, 1);
  G->status = (unsigned*)calloc((size_t)nthreads, sizeof(unsigned));
}

static unsigned grp_finish(grp_acc* G, int nthreads, int* res) {
  unsigned status = 0;
  for (int t = 0; t < nthreads; ++t) {
    status |= G->status[t];
    for (int g = 0; g < G->num_groups; ++g) {
      const size_t i = (size_t)t * G->num_groups + g;
      if (!G->touched[i]) continue;
      int* rec = res + (size_t)g * G->stride;
      rec[0] = G->keys[2 * i];
      rec[1] = G->keys[2 * i + 1];
      *(unsigned long long*)(rec + 2) += G->sums[i];
    }
  }
  free(G->keys);
  free(G->sums);
  free(G->touched);
  free(G->status);
  return status;
}

typedef struct {
  const int *od, *pk, *sk, *rev;
  const int *ht_p, *ht_s, *ht_d;
  int p_len, s_len, d_val_len;
  grp_acc G;
} q21_ctx;

static void q21_range(void* v, int tid, int64_t lo, int64_t hi) {
  q21_ctx* C = (q21_ctx*)v;
  const int ng = C->G.num_groups;
  int* keys = C->G.keys + (size_t)tid * ng * 2;
  unsigned long long* sums = C->G.sums + (size_t)tid * ng;
  unsigned char* touched = C->G.touched + (size_t)tid * ng;
  unsigned status = 0;
  for (int64_t i = lo; i < hi; ++i) {
    /* q21.cpp:106-125: part (8-byte slot, brand = upper half), supplier, date */
    int hash = C->pk[i] % C->p_len;
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    const long long p_slot = ((const long long*)C->ht_p)[hash];
    if (p_slot == 0) continue;
    const int brand = (int)(p_slot >> 32);
    hash = C->sk[i] % C->s_len;
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    if (C->ht_s[hash << 1] == 0) continue;
    hash = pht_slot(C->od[i], C->d_val_len, 19920101);
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    const int year = C->ht_d[(hash << 1) + 1];
    const int g = (int)((unsigned)brand * 7u + (unsigned)(year - 1992)) % ng;
    if (g < 0) { status |= ORC_GROUP_RANGE; continue; }
    keys[2 * g] = year;
    keys[2 * g + 1] = brand;
    sums[g] += widen(C->rev[i]);
    touched[g] = 1;
  }
  C->G.status[tid] = status;
}

unsigned orc_q21(const int* lo_orderdate, const int* lo_partkey, const int* lo_suppkey, const int* lo_revenue,
                 int64_t lo_len, const int* p_partkey, const int* p_brand1, const int* p_category, int p_len,
                 const int* d_datekey, const int* d_year, int d_len, const int* s_suppkey, const int* s_region,
                 int s_len, int d_val_len, int category, int region, int* res, int nthreads) {
  nthreads = orc_threads(nthreads);
  if (lo_len < 4096) nthreads = 1;
  int* ht_d = (int*)calloc(2 * (size_t)d_val_len, sizeof(int));
  int* ht_p = (int*)calloc(2 * (size_t)p_len, sizeof(int));
  int* ht_s = (int*)calloc(2 * (size_t)s_len, sizeof(int));
  unsigned status = build_date(d_datekey, d_year, d_len, ht_d, d_val_len);
  for (int i = 0; i < s_len; ++i) /* q21.cpp:73-82 */
    if (s_region[i] == region) {
      const int h = s_suppkey[i] % s_len;
      if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
      ht_s[h << 1] = s_suppkey[i];
    }
  for (int i = 0; i < p_len; ++i) /* q21.cpp:85-95 */
    if (p_category[i] == category) {
      const int h = p_partkey[i] % p_len;
      if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
      ht_p[h << 1] = p_partkey[i];
      ht_p[(h << 1) + 1] = p_brand1[i];
    }
  q21_ctx C = {lo_orderdate, lo_partkey, lo_suppkey, lo_revenue, ht_p, ht_s, ht_d, p_len, s_len, d_val_len};
  grp_init(&C.G, nthreads, (1998 - 1992 + 1) * 1000, 6);
  orc_parallel(lo_len, nthreads, q21_range, &C);
  status |= grp_finish(&C.G, nthreads, res);
  free(ht_d);
  free(ht_p);
  free(ht_s);
  return status;
}

typedef struct {
  const int *od, *ck, *pk, *sk, *rev, *cost;
  const int *ht_c, *ht_s, *ht_p, *ht_d;
  int c_len, s_len, p_len, d_val_len;
  grp_acc G;
} q41_ctx;

static void q41_range(void* v, int tid, int64_t lo, int64_t hi) {
  q41_ctx* C = (q41_ctx*)v;
  const int ng = C->G.num_groups;
  int* keys = C->G.keys + (size_t)tid * ng * 2;
  unsigned long long* sums = C->G.sums + (size_t)tid * ng;
  unsigned char* touched = C->G.touched + (size_t)tid * ng;
  unsigned status = 0;
  for (int64_t i = lo; i < hi; ++i) {
    /* q41.cpp:117-134: supplier, customer (-> nation), part, date (-> year) */
    int hash = C->sk[i] % C->s_len;
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    if (C->ht_s[hash << 1] == 0) continue;
    hash = C->ck[i] % C->c_len;
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    if (C->ht_c[hash << 1] == 0) continue;
    const int c_nation = C->ht_c[(hash << 1) + 1];
    hash = C->pk[i] % C->p_len;
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    if (C->ht_p[hash << 1] == 0) continue;
    hash = pht_slot(C->od[i], C->d_val_len, 19920101);
    if (hash < 0) { status |= ORC_PROBE_RANGE; continue; }
    const int year = C->ht_d[(hash << 1) + 1];
    const int g = (int)((unsigned)c_nation * 7u + (unsigned)(year - 1992)) % ng;
    if (g < 0) { status |= ORC_GROUP_RANGE; continue; }
    keys[2 * g] = year;
    keys[2 * g + 1] = c_nation;
    sums[g] += widen(i32_sub(C->rev[i], C->cost[i]));
    touched[g] = 1;
  }
  C->G.status[tid] = status;
}

unsigned orc_q41(const int* lo_orderdate, const int* lo_custkey, const int* lo_partkey, const int* lo_suppkey,
                 const int* lo_revenue, const int* lo_supplycost, int64_t lo_len, const int* d_datekey,
                 const int* d_year, int d_len, const int* p_partkey, const int* p_mfgr, int p_len,
                 const int* s_suppkey, const int* s_region, int s_len, const int* c_custkey, const int* c_region,
                 const int* c_nation, int c_len, int d_val_len, int c_region_eq, int s_region_eq, int mfgr_a,
                 int mfgr_b, int* res, int nthreads) {
  nthreads = orc_threads(nthreads);
  if (lo_len < 4096) nthreads = 1;
  int* ht_d = (int*)calloc(2 * (size_t)d_val_len, sizeof(int));
  int* ht_s = (int*)calloc(2 * (size_t)s_len, sizeof(int));
  int* ht_c = (int*)calloc(2 * (size_t)c_len, sizeof(int));
  int* ht_p = (int*)calloc(2 * (size_t)p_len, sizeof(int));
  unsigned status = build_date(d_datekey, d_year, d_len, ht_d, d_val_len);
  for (int i = 0; i < c_len; ++i) /* q41.cpp:73-83 */
    if (c_region[i] == c_region_eq) {
      const int h = c_custkey[i] % c_len;
      if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
      ht_c[h << 1] = c_custkey[i];
      ht_c[(h << 1) + 1] = c_nation[i];
    }
  for (int i = 0; i < s_len; ++i) /* q41.cpp:86-94 */
    if (s_region[i] == s_region_eq) {
      const int h = s_suppkey[i] % s_len;
      if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
      ht_s[h << 1] = s_suppkey[i];
    }
  for (int i = 0; i < p_len; ++i) /* q41.cpp:98-106 */
    if (p_mfgr[i] == mfgr_a || p_mfgr[i] == mfgr_b) {
      const int h = p_partkey[i] % p_len;
      if (h < 0) { status |= ORC_PROBE_RANGE; continue; }
      ht_p[h << 1] = p_partkey[i];
    }
  q41_ctx C = {lo_orderdate, lo_custkey, lo_partkey, lo_suppkey, lo_revenue, lo_supplycost,
               ht_c, ht_s, ht_p, ht_d, c_len, s_len, p_len, d_val_len};
  grp_init(&C.G, nthreads, (1998 - 1992 + 1) * 25, 4);
  orc_parallel(lo_len, nthreads, q41_range, &C);
  status |= grp_finish(&C.G, nthreads, res);
  free(ht_d);
  free(ht_s);
  free(ht_c);
  free(ht_p);
  return status;
}

void orc_merge(int* res_cpu, const int* res_gpu, int num_groups) {
  /* CPUProcessing.cu:1803-1807 */
  for (int i = 0; i < num_groups; ++i) {
    for (int k = 0; k < 4; ++k)
      if (res_cpu[i * 6 + k] == 0) res_cpu[i * 6 + k] = res_gpu[i * 6 + k];
    ((unsigned long long*)res_cpu)[i * 3 + 2] += ((const unsigned long long*)res_gpu)[i * 3 + 2];
  }
}
