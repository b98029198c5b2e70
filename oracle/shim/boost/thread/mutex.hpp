#pragma once
#include "../_shim_common.hpp"
#include <condition_variable>
namespace boost {
struct mutex : std::mutex { using scoped_lock = std::unique_lock<std::mutex>; };
using condition = std::condition_variable_any;
struct thread : std::thread {
    using std::thread::thread;
    static unsigned hardware_concurrency() { return std::thread::hardware_concurrency(); }
};
struct thread_group {
    std::vector<std::thread> ts;
    template <class F> void create_thread(F f) { ts.emplace_back(f); }
    void join_all() { for (auto& t : ts) t.join(); ts.clear(); }
};
template <class T> std::reference_wrapper<T> ref(T& t) { return std::ref(t); }
}  // namespace boost
