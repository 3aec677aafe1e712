#pragma once
// GraphOne's graph/graph_arch_ref.h: the same names, provided by
// graph/graph.h.
#include "GraphOne/graph/graph.h"
