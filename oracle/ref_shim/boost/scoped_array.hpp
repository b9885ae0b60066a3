// Minimal stand-in for boost::scoped_array: owns a new[]-allocated array.
#pragma once
#include <cstddef>
namespace boost {
template <typename T>
class scoped_array {
public:
    explicit scoped_array(T* p = nullptr) : p_(p) {}
    ~scoped_array() { delete[] p_; }
    scoped_array(const scoped_array&) = delete;
    scoped_array& operator=(const scoped_array&) = delete;
    T& operator[](std::ptrdiff_t i) const { return p_[i]; }
    T* get() const { return p_; }
private:
    T* p_;
};
}  // namespace boost
