#pragma once
// GraphOne's vec/dense.h: the same names, provided by
// base/buffer.h.
#include "GraphOne/base/buffer.h"
