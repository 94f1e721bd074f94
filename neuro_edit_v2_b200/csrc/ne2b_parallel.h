// ne2b_parallel.h — host-side fork/join over index ranges (admission passes).
#pragma once
#include <stdint.h>

#include <algorithm>
#include <thread>
#include <vector>

namespace ne2b {

// Split [0, n) over up to 8 host threads when n is large (synapse-sized
// loops of admission); small ranges run inline.
template <class F>
void parallel_for(uint64_t n, F f) {
    const unsigned hw = std::thread::hardware_concurrency();
    const unsigned T = std::min(8u, hw ? hw : 1u);
    if (n < (1u << 20) || T <= 1) {
        f((uint64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    const uint64_t chunk = (n + T - 1) / T;
    for (unsigned k = 0; k < T; ++k) {
        const uint64_t lo = k * chunk, hi = std::min(n, lo + chunk);
        if (lo < hi) th.emplace_back(f, lo, hi);
    }
    for (auto &x : th) x.join();
}

}  // namespace ne2b
