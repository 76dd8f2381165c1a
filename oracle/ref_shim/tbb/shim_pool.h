// std::thread stand-in for the few oneTBB entry points the reference CPU
// sources call (parallel_for over an index range, parallel_reduce, stable
// parallel_sort). Written for the oracle build only; it is not oneTBB and its
// scheduling differs (dynamic chunks from an atomic counter). parallel_sort is
// std::stable_sort, so equal keys keep their input order.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstdlib>
#include <thread>
#include <vector>

namespace tbb {

inline int shim_threads() {
    static int n = [] {
        const char* e = std::getenv("ASTER_REF_THREADS");
        int v = e ? std::atoi(e) : 0;
        if (v <= 0) v = (int)std::thread::hardware_concurrency();
        return v > 0 ? v : 1;
    }();
    return n;
}

// Runs body(lo, hi) over [first, last) split into dynamic chunks.
template <class Index, class ChunkFn>
void shim_run_chunks(Index first, Index last, ChunkFn&& body) {
    if (!(first < last)) return;
    const size_t n = (size_t)(last - first);
    const int T = std::min<size_t>((size_t)shim_threads(), n);
    if (T <= 1) { body(first, last); return; }
    const size_t chunk = std::max<size_t>(1, n / ((size_t)T * 16));
    std::atomic<size_t> next{0};
    auto worker = [&] {
        for (;;) {
            size_t lo = next.fetch_add(chunk);
            if (lo >= n) break;
            size_t hi = std::min(n, lo + chunk);
            body((Index)(first + (Index)lo), (Index)(first + (Index)hi));
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(T - 1);
    for (int t = 1; t < T; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

}  // namespace tbb
