#pragma once
// GraphOne's loader/edge_cache.h: the same names, provided by
// loader/loader.h.
#include "GraphOne/loader/loader.h"
