#pragma once
#include "shim_pool.h"

namespace tbb {
template <class Index, class Func>
void parallel_for(Index first, Index last, const Func& f) {
    shim_run_chunks(first, last, [&](Index lo, Index hi) {
        for (Index i = lo; i < hi; ++i) f(i);
    });
}
}  // namespace tbb
