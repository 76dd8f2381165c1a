#pragma once
#include <algorithm>

namespace tbb {
// Stable on purpose: ties keep input (body index) order.
template <class It, class Cmp>
void parallel_sort(It first, It last, const Cmp& cmp) { std::stable_sort(first, last, cmp); }
template <class It>
void parallel_sort(It first, It last) { std::stable_sort(first, last); }
}  // namespace tbb
