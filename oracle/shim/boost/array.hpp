#pragma once
#include "_shim_common.hpp"
namespace boost { template <class T, std::size_t N> using array = std::array<T, N>; }
