// Minimal header-only stand-ins for the handful of Boost interfaces that the
// reference's CPU sources use.  Written for the oracle build only: nothing in
// the product links against these.  Each header provides just the names the
// reference calls, with the documented Boost semantics.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <iostream>
#include <filesystem>
#include <fstream>
#include <functional>
#include <memory>
#include <mutex>
#include <optional>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
