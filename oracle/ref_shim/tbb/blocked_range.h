#pragma once
#include <cstddef>

namespace tbb {
struct split {};

template <class Value>
class blocked_range {
public:
    blocked_range(Value b, Value e) : b_(b), e_(e) {}
    Value begin() const { return b_; }
    Value end() const { return e_; }
    bool empty() const { return !(b_ < e_); }
    std::size_t size() const { return (std::size_t)(e_ - b_); }
private:
    Value b_, e_;
};
}  // namespace tbb
