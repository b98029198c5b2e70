#pragma once
// Included by the reference's vina.h and not used by its CPU search path.
#include "../_shim_common.hpp"
