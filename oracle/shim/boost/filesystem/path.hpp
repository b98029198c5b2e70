#pragma once
#include "../_shim_common.hpp"
namespace boost { namespace filesystem {
using path = std::filesystem::path;
using std::filesystem::exists;
using std::filesystem::is_directory;
using std::filesystem::create_directory;
using std::filesystem::create_directories;
using filesystem_error = std::filesystem::filesystem_error;
struct ifstream : std::ifstream {
    ifstream() = default;
    explicit ifstream(const path& p, std::ios_base::openmode m = std::ios_base::in) : std::ifstream(p, m) {}
};
struct ofstream : std::ofstream {
    ofstream() = default;
    explicit ofstream(const path& p, std::ios_base::openmode m = std::ios_base::out) : std::ofstream(p, m) {}
};
}}  // namespace boost::filesystem
