#pragma once
#include "../_shim_common.hpp"
