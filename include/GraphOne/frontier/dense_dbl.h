#pragma once
// GraphOne's frontier/dense_dbl.h: the same names, provided by
// frontier/frontier.h.
#include "GraphOne/frontier/frontier.h"
