#pragma once
#include "_shim_common.hpp"
namespace boost {
// boost::optional subset: engaged test, get(), assignment from T.
template <class T> class optional : public std::optional<T> {
public:
    using std::optional<T>::optional;
    optional(const optional&) = default;
    optional& operator=(const optional&) = default;
    optional& operator=(const T& v) { std::optional<T>::operator=(v); return *this; }
    T& get() { return this->value(); }
    const T& get() const { return this->value(); }
};
}  // namespace boost
