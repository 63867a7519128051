// Stand-in for the two TBB names common/seed_pos_table.cu uses through this
// header: tbb::blocked_range and tbb::parallel_for.  The range is split into
// grain-sized pieces handed to std::thread workers; the body's own
// __sync_fetch_and_add keeps the bucket counts correct in any order, as it
// does under TBB.  Test infrastructure for the reference harness.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <thread>
#include <vector>

namespace tbb {

template <typename T>
class blocked_range {
  public:
    blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), grain_(grain ? grain : 1) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    size_t grainsize() const { return grain_; }

  private:
    T b_, e_;
    size_t grain_;
};

template <typename T, typename Body>
void parallel_for(const blocked_range<T>& range, const Body& body) {
    const T b = range.begin(), e = range.end();
    if (e <= b) return;
    const size_t n = (size_t)(e - b);
    const size_t grain = range.grainsize();
    const size_t pieces = (n + grain - 1) / grain;
    unsigned hw = std::thread::hardware_concurrency();
    size_t workers = std::min<size_t>(pieces, hw ? hw : 1);
    std::atomic<size_t> next{0};
    auto run = [&]() {
        for (;;) {
            size_t k = next.fetch_add(1);
            if (k >= pieces) return;
            T lo = (T)(b + k * grain);
            T hi = (T)std::min<size_t>((size_t)b + (k + 1) * grain, (size_t)e);
            body(blocked_range<T>(lo, hi, grain));
        }
    };
    std::vector<std::thread> pool;
    for (size_t w = 1; w < workers; ++w) pool.emplace_back(run);
    run();
    for (auto& t : pool) t.join();
}

}  // namespace tbb
