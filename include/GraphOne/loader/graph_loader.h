#pragma once
// GraphOne's loader/graph_loader.h: the same names, provided by
// loader/loader.h.
#include "GraphOne/loader/loader.h"
