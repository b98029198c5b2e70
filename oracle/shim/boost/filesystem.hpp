#pragma once
#include "filesystem/path.hpp"
