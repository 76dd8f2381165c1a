#pragma once
#include <mutex>
#include <vector>
#include "blocked_range.h"
#include "shim_pool.h"

namespace tbb {
// Functional form: each chunk reduces from `identity`, partials are combined
// in chunk order afterwards so the result does not depend on thread timing.
template <class Value, class T, class Func, class Reduction>
T parallel_reduce(const blocked_range<Value>& range, const T& identity,
                  const Func& f, const Reduction& red) {
    std::mutex mu;
    std::vector<std::pair<Value, T>> parts;
    shim_run_chunks(range.begin(), range.end(), [&](Value lo, Value hi) {
        T part = f(blocked_range<Value>(lo, hi), identity);
        std::lock_guard<std::mutex> g(mu);
        parts.emplace_back(lo, part);
    });
    std::sort(parts.begin(), parts.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    T acc = identity;
    for (auto& p : parts) acc = red(acc, p.second);
    return acc;
}

// Imperative form: body(range) accumulates into a split copy per chunk,
// then the copies are joined in chunk order.
template <class Value, class Body>
void parallel_reduce(const blocked_range<Value>& range, Body& body) {
    std::mutex mu;
    std::vector<std::pair<Value, Body*>> parts;
    shim_run_chunks(range.begin(), range.end(), [&](Value lo, Value hi) {
        Body* b = new Body(body, split());
        (*b)(blocked_range<Value>(lo, hi));
        std::lock_guard<std::mutex> g(mu);
        parts.emplace_back(lo, b);
    });
    std::sort(parts.begin(), parts.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& p : parts) { body.join(*p.second); delete p.second; }
}
}  // namespace tbb
