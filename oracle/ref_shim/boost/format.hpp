// Minimal stand-in for boost::format: the reference's exception classes take
// one by const reference and call str(); nothing here formats.
#pragma once
#include <string>
namespace boost {
class format {
public:
    explicit format(const std::string& s = std::string()) : s_(s) {}
    template <typename T>
    format& operator%(const T&) { return *this; }
    std::string str() const { return s_; }
private:
    std::string s_;
};
}  // namespace boost
