// Test infrastructure (the oracle): a parallel loop over independent cells.
#pragma once

#include <algorithm>
#include <thread>
#include <vector>

namespace oracle_par {

// Loops over independent cells split by x-slab across the host's cores; the
// results do not depend on the thread count (no cell reads another cell's
// output of the same loop).
template <typename F>
void parallel_for(int n, F&& body) {
    const int hw = int(std::max(1u, std::thread::hardware_concurrency()));
    const int k = std::max(1, std::min(n, hw));
    if (k == 1) {
        for (int i = 0; i < n; ++i) body(i);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(size_t(k));
    for (int t = 0; t < k; ++t)
        pool.emplace_back([&, t]() {
            for (int i = t * n / k; i < (t + 1) * n / k; ++i) body(i);
        });
    for (auto& th : pool) th.join();
}

}  // namespace oracle_par
