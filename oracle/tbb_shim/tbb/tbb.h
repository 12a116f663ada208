// Minimal stand-in for the parts of oneTBB that the reference's standalone CPU engine
// (src/cpu/ssb/q*.cpp) uses: blocked_range, parallel_for and simple_partitioner.
// TEST INFRASTRUCTURE ONLY (TBB is not installed in this image). Chunks of at most the
// grain size are handed to std::threads from a shared counter, which matches TBB's
// contract for these calls (each index visited exactly once, ranges no larger than the
// grain when a simple_partitioner is given).
#pragma once
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdlib>
#include <thread>
#include <vector>

namespace tbb {

template <typename Value>
class blocked_range {
 public:
  blocked_range(Value b, Value e, std::size_t grain = 1) : b_(b), e_(e), grain_(grain ? grain : 1) {}
  Value begin() const { return b_; }
  Value end() const { return e_; }
  std::size_t size() const { return static_cast<std::size_t>(e_ - b_); }
  std::size_t grainsize() const { return grain_; }
  bool empty() const { return !(b_ < e_); }

 private:
  Value b_, e_;
  std::size_t grain_;
};

class simple_partitioner {};
class auto_partitioner {};

inline int shim_threads() {
  const char* env = std::getenv("MB_REF_THREADS");
  int n = env ? std::atoi(env) : 0;
  if (n <= 0) n = static_cast<int>(std::thread::hardware_concurrency());
  return n > 0 ? n : 1;
}

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& range, const Body& body) {
  const std::size_t n = range.size();
  if (n == 0) return;
  const std::size_t grain = range.grainsize();
  const std::size_t chunks = (n + grain - 1) / grain;
  std::atomic<std::size_t> next{0};
  auto worker = [&]() {
    for (;;) {
      const std::size_t c = next.fetch_add(1);
      if (c >= chunks) return;
      const Value b = static_cast<Value>(range.begin() + c * grain);
      const Value e = static_cast<Value>(std::min<std::size_t>(static_cast<std::size_t>(range.begin()) + (c + 1) * grain,
                                                               static_cast<std::size_t>(range.end())));
      body(blocked_range<Value>(b, e, grain));
    }
  };
  const int nt = static_cast<int>(std::min<std::size_t>(static_cast<std::size_t>(shim_threads()), chunks));
  std::vector<std::thread> ts;
  for (int t = 1; t < nt; ++t) ts.emplace_back(worker);
  worker();
  for (auto& t : ts) t.join();
}

template <typename Value, typename Body, typename Partitioner>
void parallel_for(const blocked_range<Value>& range, const Body& body, const Partitioner&) {
  parallel_for(range, body);
}

}  // namespace tbb
