#pragma once
// GraphOne's graph/builder.h: the same names, provided by
// loader/loader.h, graph/graph.h.
#include "GraphOne/loader/loader.h"
#include "GraphOne/graph/graph.h"
