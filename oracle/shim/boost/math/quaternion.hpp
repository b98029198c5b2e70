#pragma once
#include "../_shim_common.hpp"
namespace boost { namespace math {
// Quaternion a + b i + c j + d k with the operations the reference uses.
template <class T> class quaternion {
public:
    quaternion(T a = T(), T b = T(), T c = T(), T d = T()) : a(a), b(b), c(c), d(d) {}
    T R_component_1() const { return a; }
    T R_component_2() const { return b; }
    T R_component_3() const { return c; }
    T R_component_4() const { return d; }
    quaternion& operator*=(T s) { a *= s; b *= s; c *= s; d *= s; return *this; }
    quaternion& operator/=(T s) { a /= s; b /= s; c /= s; d /= s; return *this; }
    quaternion& operator*=(const quaternion& r) {  // Hamilton product
        T at = a * r.a - b * r.b - c * r.c - d * r.d;
        T bt = a * r.b + b * r.a + c * r.d - d * r.c;
        T ct = a * r.c - b * r.d + c * r.a + d * r.b;
        T dt = a * r.d + b * r.c - c * r.b + d * r.a;
        a = at; b = bt; c = ct; d = dt;
        return *this;
    }
    quaternion& operator/=(const quaternion& r) {  // this * conj(r) / |r|^2
        T den = r.a * r.a + r.b * r.b + r.c * r.c + r.d * r.d;
        quaternion conj(r.a / den, -r.b / den, -r.c / den, -r.d / den);
        return (*this) *= conj;
    }
    T a, b, c, d;
};
template <class T> quaternion<T> operator*(quaternion<T> l, const quaternion<T>& r) { return l *= r; }
template <class T> quaternion<T> operator*(quaternion<T> l, T s) { return l *= s; }
template <class T> quaternion<T> operator*(T s, quaternion<T> l) { return l *= s; }
template <class T> quaternion<T> operator/(quaternion<T> l, const quaternion<T>& r) { return l /= r; }
template <class T> quaternion<T> operator/(quaternion<T> l, T s) { return l /= s; }
// Norm with max-scaling against overflow.
template <class T> T abs(const quaternion<T>& q) {
    T m = std::max(std::max(std::abs(q.a), std::abs(q.b)), std::max(std::abs(q.c), std::abs(q.d)));
    if (m == T(0)) return m;
    T inv = T(1) / m;
    T x = q.a * inv, y = q.b * inv, z = q.c * inv, w = q.d * inv;
    return m * std::sqrt(x * x + y * y + z * z + w * w);
}
}}  // namespace boost::math
