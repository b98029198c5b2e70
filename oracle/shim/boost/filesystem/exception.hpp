#pragma once
#include "path.hpp"
