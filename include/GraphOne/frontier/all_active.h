#pragma once
// GraphOne's frontier/all_active.h: the same names, provided by
// frontier/frontier.h.
#include "GraphOne/frontier/frontier.h"
