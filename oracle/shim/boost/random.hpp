#pragma once
#include "_shim_common.hpp"
namespace boost {
using mt19937 = std::mt19937;
template <class T> struct uniform_real {
    T a, b;
    uniform_real(T a_, T b_) : a(a_), b(b_) {}
    template <class E> T operator()(E& e) { return std::uniform_real_distribution<T>(a, b)(e); }
};
template <class T> struct uniform_int {
    T a, b;
    uniform_int(T a_, T b_) : a(a_), b(b_) {}
    template <class E> T operator()(E& e) { return std::uniform_int_distribution<T>(a, b)(e); }
};
template <class T> struct normal_distribution {
    T m, s;
    normal_distribution(T m_, T s_) : m(m_), s(s_) {}
    template <class E> T operator()(E& e) { return std::normal_distribution<T>(m, s)(e); }
};
template <class Engine, class Dist> struct variate_generator {
    Engine eng;
    Dist d;
    variate_generator(Engine e, Dist dd) : eng(e), d(dd) {}
    auto operator()() { return d(eng); }
};
}  // namespace boost
