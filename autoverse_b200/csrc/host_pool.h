// Host-side parallel loop for independent per-world work (config parsing,
// kernel stencils, seed generation) of the batched engine.
#pragma once

#include <algorithm>
#include <atomic>
#include <climits>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace flp {

// Runs fn(i) for every i in [0, n) on up to min(hardware threads, 32) host
// threads, which claim items in chunks of `grain`.  Every item is attempted;
// if any call throws, the exception of the lowest failing index is rethrown
// after all threads have joined, so the error names the same item as a
// sequential loop would.
template <class F>
void parallel_for(int n, F&& fn, int grain = 4) {
    if (n <= 0) return;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int chunks = (n + grain - 1) / grain;
    const int nt = std::min({int(std::min(hw, 32u)), chunks});
    std::mutex mu;
    int bad = INT_MAX;
    std::exception_ptr err;
    auto run = [&](int i) {
        try {
            fn(i);
        } catch (...) {
            std::lock_guard<std::mutex> lk(mu);
            if (i < bad) {
                bad = i;
                err = std::current_exception();
            }
        }
    };
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) run(i);
    } else {
        std::atomic<int> next{0};
        auto worker = [&] {
            for (;;) {
                const int c = next.fetch_add(1);
                if (c >= chunks) return;
                const int e = std::min(n, (c + 1) * grain);
                for (int i = c * grain; i < e; ++i) run(i);
            }
        };
        std::vector<std::thread> pool;
        pool.reserve(nt - 1);
        try {
            for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
        } catch (...) {
            // no more threads: the ones started and this thread finish the work
        }
        worker();
        for (std::thread& t : pool) t.join();
    }
    if (err) std::rethrow_exception(err);
}

}  // namespace flp
