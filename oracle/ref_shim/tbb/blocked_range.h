// Stand-in for tbb::blocked_range: a half-open range, enough for the
// reference's (disabled) parallel functor to compile.
#pragma once
#include <cstddef>
namespace tbb {
template <typename T>
class blocked_range {
public:
    blocked_range(T b, T e) : b_(b), e_(e) {}
    T begin() const { return b_; }
    T end() const { return e_; }
private:
    T b_, e_;
};
}  // namespace tbb
