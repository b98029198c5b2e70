#pragma once
#include "../_shim_common.hpp"
namespace boost {
// Owning vector of heap objects with value semantics on copy (deep clone),
// element access by reference and sort by the element's operator<.
template <class T> class ptr_vector {
    std::vector<std::unique_ptr<T>> v;
public:
    ptr_vector() = default;
    ptr_vector(const ptr_vector& o) { for (auto& p : o.v) v.emplace_back(new T(*p)); }
    ptr_vector& operator=(const ptr_vector& o) {
        if (this != &o) { v.clear(); for (auto& p : o.v) v.emplace_back(new T(*p)); }
        return *this;
    }
    ptr_vector(ptr_vector&&) = default;
    ptr_vector& operator=(ptr_vector&&) = default;
    std::size_t size() const { return v.size(); }
    bool empty() const { return v.empty(); }
    void push_back(T* p) { v.emplace_back(p); }
    T& operator[](std::size_t i) { return *v[i]; }
    const T& operator[](std::size_t i) const { return *v[i]; }
    T& front() { return *v.front(); }
    const T& front() const { return *v.front(); }
    T& back() { return *v.back(); }
    const T& back() const { return *v.back(); }
    void clear() { v.clear(); }
    void pop_back() { v.pop_back(); }
    void resize(std::size_t n) { while (v.size() > n) v.pop_back(); }
    void sort() {
        std::stable_sort(v.begin(), v.end(), [](const std::unique_ptr<T>& x, const std::unique_ptr<T>& y) { return *x < *y; });
    }
};
}  // namespace boost
