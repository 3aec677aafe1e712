#pragma once
// GraphOne's utils.h: the same names, provided by
// utils/limits.hpp, utils/log.hpp, utils/string.hpp, utils/string_arch.h
// (under nvcc), utils/cli.hpp.
#include "GraphOne/utils/limits.hpp"
#include "GraphOne/utils/log.hpp"
#include "GraphOne/utils/string.hpp"
#ifdef __CUDACC__
#include "GraphOne/utils/string_arch.h"
#endif
#include "GraphOne/utils/cli.hpp"
