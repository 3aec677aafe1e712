#pragma once
// GraphOne's frontier/base.h: the same names, provided by
// frontier/frontier.h.
#include "GraphOne/frontier/frontier.h"
