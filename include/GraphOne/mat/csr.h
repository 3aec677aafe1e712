#pragma once
// GraphOne's mat/csr.h: the same names, provided by
// loader/loader.h.
#include "GraphOne/loader/loader.h"
