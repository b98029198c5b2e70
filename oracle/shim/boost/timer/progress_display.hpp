#pragma once
#include "../_shim_common.hpp"
namespace boost { namespace timer {
struct progress_display {
    explicit progress_display(unsigned long, std::ostream& = std::cout) {}
    unsigned long operator++() { return 0; }
    unsigned long operator+=(unsigned long) { return 0; }
};
}}  // namespace boost::timer
