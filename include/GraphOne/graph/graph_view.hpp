#pragma once
// GraphOne's graph/graph_view.hpp: the same names, provided by
// graph/graph.h.
#include "GraphOne/graph/graph.h"
