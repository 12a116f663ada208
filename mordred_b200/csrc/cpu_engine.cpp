// cpu_engine.cpp — the CPU side of the star pipeline: filtered perfect-hash builds and
// the fused filter -> chained probe -> group-by/aggregate over host-resident fact rows.
//
// This is the engine's CPU operator set (the reference's src/gpudb/CPUProcessing.cu:
// build_CPU :1034-1104, filter_probe_group_by_CPU :723-866, probe_group_by_CPU :439-568,
// filter_probe_aggr_CPU :1628-1710, and their offset-list forms) behind the same
// mb_star_args description the GPU kernels take, so a query can run part of its segments
// here and part on the GPU and the two result arrays merge by addition.
//
// Work is split into tasks of kTaskRows rows handed out by an atomic cursor to a
// persistent pool of host threads. A task walks its rows in batches of kBatch: filters
// shrink a selection vector, each probe shrinks it further and records the payloads,
// then the survivors are aggregated into the thread's private accumulators (a scalar or
// a dense group array), which are folded into the caller's result at the end. Integer
// semantics match the GPU path exactly: int32 products/differences widened to 64 bits,
// slot = (key - key_min) % slots in 32-bit arithmetic, group index in 32-bit arithmetic.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "mordred_b200.h"

namespace mb {
namespace {

constexpr int64_t kTaskRows = 1 << 16;
constexpr int kBatch = 256;

// ---- persistent worker pool ------------------------------------------------------------
class Pool {
 public:
  static Pool& get() {
    static Pool p;
    return p;
  }
  int size() const { return static_cast<int>(workers_.size()) + 1; }

  // Run fn(worker index) on `n` workers (the caller is worker 0); returns when all end.
  void run(int n, const std::function<void(int)>& fn) {
    n = std::max(1, std::min(n, size()));
    if (n == 1) {
      fn(0);
      return;
    }
    std::unique_lock<std::mutex> call(call_mu_);  // one parallel region at a time
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      active_ = n - 1;
      pending_ = n - 1;
      ++generation_;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return pending_ == 0; });
    fn_ = nullptr;
  }

 private:
  Pool() {
    unsigned hc = std::thread::hardware_concurrency();
    const int n = hc > 1 ? static_cast<int>(hc) - 1 : 0;
    for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { loop(i + 1); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void loop(int idx) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int)>* fn;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
        if (idx > active_) continue;  // not needed in this region
        fn = fn_;
      }
      (*fn)(idx);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_cv_.notify_all();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex mu_, call_mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* fn_ = nullptr;
  uint64_t generation_ = 0;
  int active_ = 0, pending_ = 0;
  bool stop_ = false;
};

int threads_for(int requested, int64_t rows) {
  int n = requested > 0 ? requested : Pool::get().size();
  const int64_t tasks = (rows + kTaskRows - 1) / kTaskRows;
  if (tasks < n) n = static_cast<int>(std::max<int64_t>(1, tasks));
  return n;
}

inline int wrap_sub(int a, int b) { return static_cast<int>(static_cast<unsigned>(a) - static_cast<unsigned>(b)); }
inline int wrap_mul(int a, int b) { return static_cast<int>(static_cast<unsigned>(a) * static_cast<unsigned>(b)); }

struct Acc {
  unsigned long long scalar = 0, count = 0;
  unsigned status = 0;
  std::vector<unsigned long long> sums;  // per group
  std::vector<int> keys;                 // per group, 4 payload slots
  std::vector<unsigned char> touched;
};

inline bool pass_filter(int x, int mode, int c1, int c2) {
  return mode == MB_FILTER_BETWEEN ? (x >= c1 && x <= c2) : mode == MB_FILTER_EQ ? x == c1 : (x == c1 || x == c2);
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_cpu_threads(void) { return Pool::get().size(); }

extern "C" int mb_cpu_build_pht(const int* filter_col, int filter_mode, int c1, int c2, const int* dim_key,
                                const int* dim_val, int num_tuples, int* ht, int num_slots, int key_min,
                                int layout, int nthreads, unsigned int* status) {
  if (num_tuples == 0) return MB_OK;
  if (dim_key == nullptr || ht == nullptr || num_tuples < 0 || num_slots <= 0) return MB_ERR_ARG;
  if (layout != MB_HT_KEY && layout != MB_HT_KEY_VAL && layout != MB_HT_VAL_OFF) return MB_ERR_ARG;
  if (layout != MB_HT_KEY && dim_val == nullptr) return MB_ERR_ARG;
  if (filter_col && (filter_mode < MB_FILTER_EQ || filter_mode > MB_FILTER_EQ_OR_EQ)) return MB_ERR_ARG;
  const int n = threads_for(nthreads, num_tuples);
  std::atomic<unsigned> st{0};
  const int64_t chunk = (num_tuples + n - 1) / n;
  Pool::get().run(n, [&](int t) {
    const int64_t lo = t * chunk, hi = std::min<int64_t>(num_tuples, lo + chunk);
    unsigned bad = 0;
    for (int64_t i = lo; i < hi; ++i) {
      if (filter_col && !pass_filter(filter_col[i], filter_mode, c1, c2)) continue;
      const int h = wrap_sub(dim_key[i], key_min) % num_slots;
      if (h < 0) {
        bad |= MB_STATUS_PROBE_RANGE;
        continue;
      }
      // keys are unique, so every slot has one writer: plain stores suffice
      if (layout == MB_HT_KEY) {
        ht[h] = dim_key[i];
      } else if (layout == MB_HT_KEY_VAL) {
        ht[2 * static_cast<int64_t>(h)] = dim_key[i];
        ht[2 * static_cast<int64_t>(h) + 1] = dim_val[i];
      } else {
        ht[2 * static_cast<int64_t>(h)] = dim_val[i];
        ht[2 * static_cast<int64_t>(h) + 1] = static_cast<int>(i + 1);
      }
    }
    if (bad) st.fetch_or(bad);
  });
  if (status) *status |= st.load();
  return MB_OK;
}

// Fused star pipeline over host columns. Rows are the call's virtual rows [0, num_rows):
// with segment_size > 0 virtual row r reads physical row seg * segment_size + r %
// segment_size, seg = segment_group[r / segment_size] (or (start_offset + r) /
// segment_size without a list). With `rows` non-NULL only the listed virtual rows are
// processed (an offset list handed over from a GPU selection).
extern "C" int mb_cpu_star_query(const mb_star_args* a, const int* rows, int64_t num_listed, int nthreads,
                                 unsigned int* status) {
  if (a == nullptr) return MB_ERR_ARG;
  if (a->gpu_cache != nullptr) return MB_ERR_ARG;  // host columns only
  if (a->num_filters < 0 || a->num_filters > MB_MAX_FILTERS || a->num_probes < 0 || a->num_probes > MB_MAX_PROBES)
    return MB_ERR_ARG;
  if (a->res_layout < MB_RES_SCALAR || a->res_layout > MB_RES_DENSE || a->res == nullptr) return MB_ERR_ARG;
  if (a->agg_op < MB_AGG_SUM || a->agg_op > MB_AGG_MUL_PAYLOAD || a->aggr[0] == nullptr) return MB_ERR_ARG;
  if ((a->agg_op == MB_AGG_SUB || a->agg_op == MB_AGG_MUL) && a->aggr[1] == nullptr) return MB_ERR_ARG;
  if (a->agg_op == MB_AGG_MUL_PAYLOAD && (a->num_probes < 1 || a->probe[0].layout == MB_HT_KEY)) return MB_ERR_ARG;
  if (a->res_layout != MB_RES_SCALAR && a->total_val <= 0) return MB_ERR_ARG;
  if (a->segment_size < 0 || (a->segment_size > 0 && (a->segment_size & (a->segment_size - 1)) != 0))
    return MB_ERR_ARG;
  for (int f = 0; f < a->num_filters; ++f)
    if (a->filter[f].col == nullptr || a->filter[f].mode < MB_FILTER_EQ || a->filter[f].mode > MB_FILTER_EQ_OR_EQ)
      return MB_ERR_ARG;
  for (int p = 0; p < a->num_probes; ++p)
    if (a->probe[p].fkey == nullptr || a->probe[p].ht == nullptr || a->probe[p].num_slots <= 0 ||
        a->probe[p].layout < MB_HT_KEY || a->probe[p].layout > MB_HT_VAL_OFF)
      return MB_ERR_ARG;
  const int64_t total = rows ? num_listed : a->num_rows;
  if (total < 0) return MB_ERR_ARG;
  if (total == 0) return MB_OK;

  const int layout = a->res_layout, G = layout == MB_RES_SCALAR ? 1 : a->total_val;
  const int nt = threads_for(nthreads, total);
  std::vector<Acc> acc(nt);
  std::atomic<int64_t> cursor{0};
  const int64_t S = a->segment_size;
  const int shift = S > 0 ? __builtin_ctzll(static_cast<unsigned long long>(S)) : 0;

  Pool::get().run(nt, [&](int t) {
    Acc& A = acc[t];
    if (layout != MB_RES_SCALAR) {
      A.sums.assign(G, 0ull);
      A.touched.assign(G, 0);
      if (layout != MB_RES_DENSE) A.keys.assign(static_cast<size_t>(G) * 4, 0);
    }
    int64_t sel[kBatch];
    int gv[MB_MAX_PROBES][kBatch];
    for (;;) {
      const int64_t t0 = cursor.fetch_add(kTaskRows);
      if (t0 >= total) break;
      const int64_t t1 = std::min(total, t0 + kTaskRows);
      for (int64_t b0 = t0; b0 < t1; b0 += kBatch) {
        const int nb = static_cast<int>(std::min<int64_t>(kBatch, t1 - b0));
        // physical rows of the batch
        int ns = 0;
        for (int i = 0; i < nb; ++i) {
          const int64_t v = rows ? rows[b0 + i] : b0 + i;
          int64_t r = v;
          if (S > 0) {
            const int64_t seg = a->segment_group ? a->segment_group[v >> shift] : (a->start_offset + v) >> shift;
            r = (seg << shift) + (v & (S - 1));
          }
          sel[ns++] = r;
        }
        // filters, in order (count_after = f counts rows reaching filter f)
        for (int f = 0; f < a->num_filters; ++f) {
          if (a->count_after == f) A.count += ns;
          const int* col = a->filter[f].col;
          const int m = a->filter[f].mode, c1 = a->filter[f].c1, c2 = a->filter[f].c2;
          int k = 0;
          for (int i = 0; i < ns; ++i) {
            const int64_t r = sel[i];
            sel[k] = r;
            k += pass_filter(col[r], m, c1, c2);
          }
          ns = k;
        }
        if (a->count_after >= a->num_filters) A.count += ns;
        // probes, in order; payloads kept beside the selection
        int np_done = 0;
        for (int p = 0; p < a->num_probes; ++p) {
          const mb_probe& Q = a->probe[p];
          int k = 0;
          for (int i = 0; i < ns; ++i) {
            const int64_t r = sel[i];
            const int h = wrap_sub(Q.fkey[r], Q.key_min) % Q.num_slots;
            if (h < 0) {
              A.status |= MB_STATUS_PROBE_RANGE;
              continue;
            }
            int payload = 0;
            bool hit;
            if (Q.layout == MB_HT_KEY) {
              hit = Q.ht[h] != 0;
            } else {
              const int lo32 = Q.ht[2 * static_cast<int64_t>(h)], hi32 = Q.ht[2 * static_cast<int64_t>(h) + 1];
              hit = (lo32 | hi32) != 0;
              payload = Q.layout == MB_HT_KEY_VAL ? hi32 : lo32;
            }
            if (!hit) continue;
            sel[k] = r;
            for (int q = 0; q < np_done; ++q) gv[q][k] = gv[q][i];
            gv[p][k] = payload;
            ++k;
          }
          ns = k;
          ++np_done;
        }
        if (a->count_after < 0) A.count += ns;
        // aggregate
        for (int i = 0; i < ns; ++i) {
          const int64_t r = sel[i];
          const int a0 = a->aggr[0][r];
          int v;
          switch (a->agg_op) {
            case MB_AGG_SUM: v = a0; break;
            case MB_AGG_SUB: v = wrap_sub(a0, a->aggr[1][r]); break;
            case MB_AGG_MUL: v = wrap_mul(a0, a->aggr[1][r]); break;
            default: v = wrap_mul(a0, gv[0][i]); break;
          }
          const unsigned long long w = static_cast<unsigned long long>(static_cast<long long>(v));
          if (layout == MB_RES_SCALAR) {
            A.scalar += w;
            continue;
          }
          unsigned hh = static_cast<unsigned>(a->group_bias);
          for (int p = 0; p < a->num_probes; ++p)
            hh += static_cast<unsigned>(wrap_sub(gv[p][i], a->probe[p].min_val)) *
                  static_cast<unsigned>(a->probe[p].unique_val);
          const int g = static_cast<int>(hh) % a->total_val;
          if (g < 0) {
            A.status |= MB_STATUS_GROUP_RANGE;
            continue;
          }
          A.sums[g] += w;
          A.touched[g] = 1;
          if (layout != MB_RES_DENSE)
            for (int p = 0; p < a->num_probes; ++p)
              if (a->probe[p].res_slot >= 0) A.keys[static_cast<size_t>(g) * 4 + a->probe[p].res_slot] = gv[p][i];
        }
      }
    }
  });

  // fold the thread partials into the caller's result
  unsigned st = 0;
  unsigned long long scalar = 0, count = 0;
  for (const Acc& A : acc) {
    st |= A.status;
    scalar += A.scalar;
    count += A.count;
  }
  if (layout == MB_RES_SCALAR) {
    *static_cast<unsigned long long*>(a->res) += scalar;
  } else {
    const int R = layout == MB_RES_ENGINE6 ? 6 : layout == MB_RES_CRYSTAL4 ? 4 : 2;
    const int so = layout == MB_RES_ENGINE6 ? 4 : layout == MB_RES_CRYSTAL4 ? 2 : 0;
    int* res = static_cast<int*>(a->res);
    for (const Acc& A : acc)
      for (int g = 0; g < G; ++g) {
        if (!A.touched[g]) continue;
        int* dst = res + static_cast<size_t>(g) * R;
        if (layout != MB_RES_DENSE)
          for (int p = 0; p < a->num_probes; ++p) {
            const int slot = a->probe[p].res_slot;
            if (slot >= 0 && slot < so) dst[slot] = A.keys[static_cast<size_t>(g) * 4 + slot];
          }
        unsigned long long s;
        memcpy(&s, dst + so, 8);
        s += A.sums[g];
        memcpy(dst + so, &s, 8);
      }
  }
  if (a->count) *a->count += count;
  if (status) *status |= st;
  return MB_OK;
}

// Selection with compaction on the host: the rows of the call (virtual rows, or the listed
// ones) passing a's filters and probes, as an offset list in row order — the CPU operators
// filter_CPU / filter_probe_CPU / probe_CPU and their list forms (CPUProcessing.cu:3-437,
// 1158-1333). lo_off[k] = physical row; dim_off[p] (optional) = probe p's output: the
// dimension row ht[2h+1] - 1 (VAL_OFF), the payload (KEY_VAL) or 0 (KEY). This is the CPU
// half of a split query whose aggregation runs on the GPU over the list (the GPU3 forms).
extern "C" int mb_cpu_star_select(const mb_star_args* a, const int* rows, int64_t num_listed, int* lo_off,
                                  int* const* dim_off, int64_t capacity, int64_t* total_out, int nthreads,
                                  unsigned int* status) {
  if (a == nullptr || total_out == nullptr || capacity < 0) return MB_ERR_ARG;
  if (a->gpu_cache != nullptr) return MB_ERR_ARG;
  if (a->num_filters < 0 || a->num_filters > MB_MAX_FILTERS || a->num_probes < 0 || a->num_probes > MB_MAX_PROBES)
    return MB_ERR_ARG;
  if (a->segment_size < 0 || (a->segment_size > 0 && (a->segment_size & (a->segment_size - 1)) != 0))
    return MB_ERR_ARG;
  for (int f = 0; f < a->num_filters; ++f)
    if (a->filter[f].col == nullptr || a->filter[f].mode < MB_FILTER_EQ || a->filter[f].mode > MB_FILTER_EQ_OR_EQ)
      return MB_ERR_ARG;
  for (int p = 0; p < a->num_probes; ++p)
    if (a->probe[p].fkey == nullptr || a->probe[p].ht == nullptr || a->probe[p].num_slots <= 0 ||
        a->probe[p].layout < MB_HT_KEY || a->probe[p].layout > MB_HT_VAL_OFF)
      return MB_ERR_ARG;
  const int64_t total = rows ? num_listed : a->num_rows;
  if (total < 0) return MB_ERR_ARG;
  *total_out = 0;
  if (total == 0) return MB_OK;
  if (capacity > 0 && lo_off == nullptr) return MB_ERR_ARG;

  const int64_t ntasks = (total + kTaskRows - 1) / kTaskRows;
  const int nt = threads_for(nthreads, total);
  // per task: its survivors' physical rows and probe outputs, concatenated in task order
  std::vector<std::vector<int>> t_rows(ntasks), t_dims(ntasks);
  std::vector<unsigned> t_status(nt, 0);
  std::atomic<int64_t> cursor{0};
  const int64_t S = a->segment_size;
  const int shift = S > 0 ? __builtin_ctzll(static_cast<unsigned long long>(S)) : 0;
  const int np = a->num_probes;

  Pool::get().run(nt, [&](int t) {
    int64_t sel[kBatch];
    int out[MB_MAX_PROBES][kBatch];
    for (;;) {
      const int64_t t0 = cursor.fetch_add(kTaskRows);
      if (t0 >= total) break;
      const int64_t task = t0 / kTaskRows;
      const int64_t t1 = std::min(total, t0 + kTaskRows);
      std::vector<int>& tr = t_rows[task];
      std::vector<int>& td = t_dims[task];
      for (int64_t b0 = t0; b0 < t1; b0 += kBatch) {
        const int nb = static_cast<int>(std::min<int64_t>(kBatch, t1 - b0));
        int ns = 0;
        for (int i = 0; i < nb; ++i) {
          const int64_t v = rows ? rows[b0 + i] : b0 + i;
          int64_t r = v;
          if (S > 0) {
            const int64_t seg = a->segment_group ? a->segment_group[v >> shift] : (a->start_offset + v) >> shift;
            r = (seg << shift) + (v & (S - 1));
          }
          sel[ns++] = r;
        }
        for (int f = 0; f < a->num_filters; ++f) {
          const int* col = a->filter[f].col;
          const int m = a->filter[f].mode, c1 = a->filter[f].c1, c2 = a->filter[f].c2;
          int k = 0;
          for (int i = 0; i < ns; ++i) {
            const int64_t r = sel[i];
            sel[k] = r;
            k += pass_filter(col[r], m, c1, c2);
          }
          ns = k;
        }
        for (int p = 0; p < np; ++p) {
          const mb_probe& Q = a->probe[p];
          int k = 0;
          for (int i = 0; i < ns; ++i) {
            const int64_t r = sel[i];
            const int h = wrap_sub(Q.fkey[r], Q.key_min) % Q.num_slots;
            if (h < 0) {
              t_status[t] |= MB_STATUS_PROBE_RANGE;
              continue;
            }
            int o = 0;
            bool hit;
            if (Q.layout == MB_HT_KEY) {
              hit = Q.ht[h] != 0;
            } else {
              const int lo32 = Q.ht[2 * static_cast<int64_t>(h)], hi32 = Q.ht[2 * static_cast<int64_t>(h) + 1];
              if (Q.layout == MB_HT_VAL_OFF) {
                hit = (lo32 | hi32) != 0;
                o = hi32 - 1;
              } else {
                hit = (lo32 | hi32) != 0;
                o = hi32;
              }
            }
            if (!hit) continue;
            sel[k] = r;
            for (int q = 0; q < p; ++q) out[q][k] = out[q][i];
            out[p][k] = o;
            ++k;
          }
          ns = k;
        }
        for (int i = 0; i < ns; ++i) {
          tr.push_back(static_cast<int>(sel[i]));
          for (int p = 0; p < np; ++p) td.push_back(out[p][i]);
        }
      }
    }
  });
  unsigned st = 0;
  for (unsigned s : t_status) st |= s;
  int64_t k = 0;
  for (int64_t task = 0; task < ntasks; ++task) {
    const std::vector<int>& tr = t_rows[task];
    const std::vector<int>& td = t_dims[task];
    for (size_t i = 0; i < tr.size(); ++i, ++k) {
      if (k >= capacity) continue;
      lo_off[k] = tr[i];
      if (dim_off)
        for (int p = 0; p < np; ++p)
          if (dim_off[p]) dim_off[p][k] = td[i * np + p];
    }
  }
  if (k > capacity) st |= MB_STATUS_OVERFLOW;
  *total_out = k;
  if (status) *status |= st;
  return MB_OK;
}
