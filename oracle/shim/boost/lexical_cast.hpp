#pragma once
#include "_shim_common.hpp"
namespace boost {
struct bad_lexical_cast : std::bad_cast {};
// Whole-string conversion; any leftover characters or a failed read throw.
template <class T, class S> T lexical_cast(const S& s) {
    std::ostringstream os;
    os << s;
    std::istringstream in(os.str());
    T out;
    in >> out;
    if (in.fail()) throw bad_lexical_cast();
    char c;
    if (in >> c) throw bad_lexical_cast();
    return out;
}
template <> inline std::string lexical_cast<std::string, unsigned>(const unsigned& s) { return std::to_string(s); }
}  // namespace boost
